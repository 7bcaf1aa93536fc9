/*
 * pyfwi_b200 -- C ABI of the B200 elastic propagator and adjoint gradient.
 *
 * This is the native boundary under the Python drop-in for PyFWI's hot path
 * (PyFWI src/PyFWI/wave_propagation.py: WavePropagator.forward_modeling and
 * WavePropagator.gradient).  In the reference that boundary is a set of
 * OpenCL kernels launched through pyopencl once per time step and shot
 * (wave_propagation.py:625-856); here one call runs every time step of every
 * shot on the device.
 *
 * Conventions
 *  - Every function returns an int status: PYFWI_OK (0) or a negative code;
 *    pyfwi_last_error() gives the message of the calling thread's last error.
 *  - All array arguments except those marked "host" are device pointers.
 *    The caller owns all device memory: inputs, outputs and one workspace of
 *    pyfwi_workspace_size() bytes (256-byte aligned).  No call allocates or
 *    frees device memory.
 *  - `stream` is a cudaStream_t passed as void*.  Calls only enqueue work on
 *    it (plus small host-to-device copies of constants on the same stream);
 *    they do not synchronise except where stated.
 *  - A plan is not thread-safe: use one plan per host thread/stream.
 *  - Grid coordinates: the padded grid has nz + 2*npml rows (z) and
 *    nx + 2*npml columns (x); cell (i, j) is row i, column j.
 */
#ifndef PYFWI_B200_H
#define PYFWI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PYFWI_ABI_VERSION 8

/* The most kernel launches a call replays as one CUDA graph (options.graph);
 * calls with more launch directly. */
#define PYFWI_GRAPH_MAX_LAUNCHES 600000LL

enum pyfwi_status {
    PYFWI_OK = 0,
    PYFWI_E_INVALID = -1,   /* bad argument or geometry */
    PYFWI_E_WORKSPACE = -2, /* workspace missing or smaller than required */
    PYFWI_E_CUDA = -3,      /* a CUDA runtime call failed */
    PYFWI_E_TIMEOUT = -4,   /* a bounded device-side wait gave up */
    PYFWI_E_STATE = -5      /* call out of order (e.g. gradient before forward) */
};

enum pyfwi_checkpoint {
    /* Exact: the adjoint sees the forward state of every step, stored or
     * recomputed from restart states; identical to the reference with
     * chpr = 100 (wave_propagation.py:95-100, 710-727, 761-779). */
    PYFWI_CKPT_EXACT = 0,
    /* The reference's chpr < 100 scheme: states stored at the listed steps,
     * the rest rebuilt by reverse-time steps (wave_propagation.py:761-812). */
    PYFWI_CKPT_REVERSE = 1
};

/* Format of the stored forward states the imaging reads (exact mode): FP32;
 * BF16 (8 mantissa bits, half the store); or 24 bits (the float rounded to
 * 15 mantissa bits, kept as a BF16 plane plus a byte plane: three quarters
 * of the store).  The forward recurrence is FP32 in every format. */
enum pyfwi_snapshot { PYFWI_SNAP_FP32 = 0, PYFWI_SNAP_BF16 = 1, PYFWI_SNAP_FP24 = 2 };

enum pyfwi_parameterization { PYFWI_PARAM_LMD = 0, PYFWI_PARAM_DV = 1 };

/* One straight line of receivers.  Receiver k (0 <= k < count) sits at cell
 * (row0 + k*drow, col0 + k*dcol) and fills trace slot slot0 + k.  The three
 * receiver groups of the reference kernels (elastic_surface.cl:30-39,
 * elastic_crosswell.cl:95-102, elastic.cl:65-96) are each one line. */
typedef struct pyfwi_rec_line {
    int32_t row0, col0;
    int32_t drow, dcol;
    int32_t count;
    int32_t slot0;
    int32_t vz_from_vx; /* 1: the vz trace records vx (elastic_crosswell.cl:98) */
} pyfwi_rec_line;

/* Survey geometry.  Mirrors the compile-time macros the reference builds per
 * WavePropagator (wave_propagation.py:423-490) plus the per-shot source cells
 * (wave_propagation.py:86-87). */
typedef struct pyfwi_geometry {
    int32_t nz, nx;         /* model grid, without the absorbing layer */
    int32_t npml;           /* absorbing-layer width in cells */
    int32_t half_order;     /* sdo: 2 (4th-order stencil) or 4 (8th) */
    int32_t nt;             /* internal time steps */
    int32_t nt_ext;         /* trace samples */
    int32_t dt_scale;       /* internal steps per trace sample */
    float dt;               /* internal step (s) */
    float dh;               /* cell size (m) */
    float c[4];             /* stencil coefficients c1..c4 */
    int32_t ns;             /* shots */
    int32_t nr;             /* trace slots per shot */
    int32_t n_lines;        /* receiver lines, 1..3 */
    pyfwi_rec_line lines[3];
    /* Gradient window in model-grid cells, [row0,row1) x [col0,col1): the
     * region gradient_reading keeps (wave_propagation.py:303-318). */
    int32_t mask_row0, mask_row1, mask_col0, mask_col1;
} pyfwi_geometry;

/* Run options. */
/* Which gradient pyfwi_gradient computes.
 * REFERENCE: PyFWI's adjoint-state gradient (Adj_update_tau, Adj_update_v,
 *   Grad: elastic.cl:372-526; wave_propagation.py:751-938), masked and
 *   normalised by gradient_reading.
 * EXACT: no counterpart in the reference: the exact derivative of
 *   J = 1/2 sum (trace - observed)^2 of the discrete forward step of this
 *   library (transposed step, the absorbing profiles held fixed), on the whole
 *   model grid with no mask; the residual planes are dJ/dtrace per raw trace.
 *   Needs PYFWI_CKPT_EXACT and no energy terms; with PYFWI_SNAP_BF16 or
 *   PYFWI_SNAP_FP24 the transposed step reads S_{t+1} and S_t from the
 *   snapshots. */
enum pyfwi_adjoint { PYFWI_ADJOINT_REFERENCE = 0, PYFWI_ADJOINT_EXACT = 1 };

typedef struct pyfwi_options {
    int32_t checkpoint;     /* enum pyfwi_checkpoint */
    int32_t segment;        /* exact mode: steps per recompute segment; 0 = all steps */
    int32_t snapshot;       /* exact mode: enum pyfwi_snapshot for the imaged states */
    int32_t shot_batch;     /* shots propagated together; 0 = all */
    int32_t energy;         /* 1: also accumulate the energy terms (energy_balancing) */
    int32_t nchp;           /* reverse mode: number of checkpoint steps */
    const int32_t *chp;     /* host; reverse mode: the checkpoint steps (copied) */
    int32_t tile;           /* kernel variant (see pyfwi_tile_count): 0..2 tile kernels with
                               16 / 8 / 32 rows per tile, 3..5 streaming kernels with
                               128 / 64 / 256 columns per CTA, 6..7 16-row tile kernels
                               whose adjoint CTAs carry 2 / 4 shots (forward as 0),
                               8..10 tile kernels of 16 / 8 / 32 rows with the forward
                               tile staged by TMA box copies (adjoint as 0..2), 11 the
                               16-row tile kernels whose adjoint prefetches the tile's
                               gradient accumulators into shared memory */
    int32_t graph;          /* 1: replay time loops as CUDA graphs (calls of more than
                               PYFWI_GRAPH_MAX_LAUNCHES kernel launches run directly) */
    int32_t chunk;          /* streaming kernels: grid rows per CTA, 0 = from the grid size */
    int32_t adj_tile;       /* adjoint+imaging step variant + 1 (same numbering as tile); 0 = tile */
    int32_t adjoint;        /* enum pyfwi_adjoint */
    int32_t persist;        /* 1: run the time loops of small surveys as persistent cooperative
                               kernels (many steps per launch, a grid barrier between steps)
                               where the layout allows: exact checkpoints holding every step in
                               FP32, the tile kernels (variants 0..2), the reference adjoint;
                               otherwise (and inside a caller's stream capture) one launch per step */
    int32_t overlap;        /* 1: exact checkpoints in FP32 with recompute segments: recompute
                               segment m-1 on a second stream of the plan while the adjoint of
                               segment m runs (two segment buffers in the workspace) */
    int32_t store_diffs;    /* 1: exact checkpoints in FP32, reference adjoint without energy
                               terms, tile kernels 0..2: the forward steps that fill the segment
                               store write the five differences of each state that the imaging
                               reads (Dx+ vx, Dz- vz, Dz+ vz + Dx- vz, Dx- txx + Dz- txz,
                               Dz+ tzz + Dx+ txz) in place of the state, and the adjoint step
                               reads them instead of differencing the state; the recurrence
                               runs in the two work states.  Same store size; otherwise ignored */
} pyfwi_options;

typedef struct pyfwi_plan pyfwi_plan;

/* Build a plan.  srcx, srcz: host arrays of ns padded-grid source cells
 * (replaces WavePreparation.__init__, wave_propagation.py:18-246, on the
 * native side).  Allocates host memory only. */
int pyfwi_plan_create(const pyfwi_geometry *geom, const int32_t *srcx, const int32_t *srcz,
                      const pyfwi_options *opt, pyfwi_plan **plan);
int pyfwi_plan_destroy(pyfwi_plan *plan);

/* Bytes of device workspace the plan needs. */
int pyfwi_workspace_size(const pyfwi_plan *plan, size_t *bytes);

/* Load a model into the workspace: pad by edge replication, form
 * mu = rho*vs^2, lam = rho*vp^2 - 2*mu, buoyancy 1/rho, and scale the
 * damping profiles by max(vp).  Replaces expand_model (fwi_tools.py:776-811),
 * pml_preparation (wave_propagation.py:400-407) and elastic_buffers
 * (wave_propagation.py:570-591).
 *   vp, vs, rho   [nz][nx] float32
 *   damp_x        [nx + 2*npml] damping profile per column (before the vp_max factor)
 *   damp_z        [nz + 2*npml] damping profile per row */
int pyfwi_set_model(pyfwi_plan *plan, void *workspace, size_t workspace_bytes, const float *vp,
                    const float *vs, const float *rho, const float *damp_x, const float *damp_z, void *stream);

/* Forward modelling of every shot.  Replaces forward_propagator and its
 * per-step loop (wave_propagation.py:625-733).
 *   src_vals  host [n_src][4]: (vx, vz, taux, tauz) amplitudes added at the
 *             source cell on injection k; injections past n_src add zero
 *   traces    [5][nt_ext][ns*nr]: vx, vz, taux, tauz, tauxz; column s*nr + r
 *             is receiver slot r of shot s (the reference's '2d' layout) */
int pyfwi_forward(pyfwi_plan *plan, void *workspace, size_t workspace_bytes, const float *src_vals,
                  int32_t n_src, float *traces, void *stream);

/* Adjoint-state gradient for the last forward call's model and sources.
 * Replaces __adjoint_modelling_per_source, __kernel_gradient and
 * gradient_reading + grad_lmd_to_vd (wave_propagation.py:735-856, 279-331,
 * grad_switcher.py:331-383).
 *   residual  5 device pointers (vx, vz, taux, tauz, tauxz), each
 *             [nt_ext][ns*nr]; NULL means an all-zero component
 *   grad      [3][nz][nx]: (lam, mu, rho) or (vp, vs, rho) per `parameterization`
 *   raw       optional [6][nz+2npml][nx+2npml]: the accumulators
 *             (Gmu, Glam, Grho, and the three energy terms) before masking */
int pyfwi_gradient(pyfwi_plan *plan, void *workspace, size_t workspace_bytes, const float *const *residual,
                   int32_t parameterization, float *grad, float *raw, void *stream);

/* Doubles of scratch a reduction needs (pyfwi_l2_residual): one partial sum
 * per block of the reduction grid. */
#define PYFWI_REDUCE_SLOTS 2368

/* L2 misfit and residual (CostFunction.l2, fwi_tools.py:1402-1422):
 * res = est - obs (float32), *misfit += 0.5 * sum(res^2) (float64 sum on
 * device).  scratch: PYFWI_REDUCE_SLOTS device doubles for the per-block
 * partial sums, added in a fixed order: the same inputs give the same bits. */
int pyfwi_l2_residual(const float *est, const float *obs, float *res, int64_t n, double *scratch, double *misfit,
                      void *stream);

/* One misfit-and-gradient evaluation, the work of FWI.fprime (fwi.py:
 * 229-246: forward_modeling, CostFunction.l2 on the section, gradient) fused
 * per shot group: each group is modelled once, its L2 residual against the
 * observed traces is formed on the device, and its adjoint runs while its
 * forward states are still stored.  pyfwi_set_model must come first.
 * observed[5]: device [nt_ext][ns*nr] observed traces per field in the
 *   '2d' section layout, NULL for a field not in the misfit.  mean_stress = 1
 *   for components 0: the txx and tzz slots then hold the observed 'taux' and
 *   'tauz' sections, both compared with (txx + tzz) / 2.
 * adjoint_source[5]: device [nt_ext][ns*nr] buffers receiving the adjoint
 *   sources (the section residuals; for PYFWI_ADJOINT_EXACT with
 *   mean_stress, half their sum in both stress slots); needed where observed
 *   is set (both stress slots with mean_stress).
 * traces: device [5][nt_ext][ns*nr], receives the modelled traces.
 * misfit: device double, receives sum over the section keys of
 *   0.5 * |modelled - observed|^2 (accumulated in double).
 * Not for surveys whose section reorders traces (acquisition 2 with well
 * receivers): use pyfwi_forward + pyfwi_gradient there. */
int pyfwi_misfit_gradient(pyfwi_plan *plan, void *workspace, size_t bytes, const float *src_vals, int32_t n_src,
                          const float *const *observed, int32_t mean_stress, float *const *adjoint_source,
                          int32_t parameterization, float *traces, float *grad, double *misfit, void *stream);

/* Low-pass filter of the multiscale misfit (lowpass / adj_lowpass,
 * fwi_tools.py:1188-1258): every trace (column) of n_planes device planes
 * [nt][ncols] (time along rows) is convolved along time with the filter's
 * symmetric impulse response g, y[t] = sum_s g[|t - s|] x[s], by FFTs of
 * nfft points on the device.
 *   filter  device float[2 * nfft]: the real spectrum of the response
 *           embedded in a circulant of nfft points, 1/nfft included
 *           (filter[0..nfft)), then the twiddles exp(-2 pi i j / nfft),
 *           j < nfft / 2, as (cos, sin) pairs; built on the host from the
 *           Butterworth design (pyfwi_b200.fwi_tools.lowpass_spectrum)
 *   nfft    a power of two with 2 nt - 1 <= nfft <= 16384 (nt <= 8192)
 * in and out must not overlap.  Allocates nothing; one kernel launch. */
int pyfwi_lowpass(const float *filter, int32_t nfft, const float *in, float *out, int32_t nt, int64_t ncols,
                  int32_t n_planes, void *stream);

/* Trace section (acquisition.py:313-333): out = (a + b) / 2 elementwise. */
int pyfwi_mean2(const float *a, const float *b, float *out, int64_t n, void *stream);

/* Gradient smoothing (the gaussian_filter(g, g_smooth) calls of
 * wave_propagation.py:923-936): n stacked (nz, nx) device arrays are
 * correlated along z, then along x, with the 2*radius+1 host weights
 * (normalised Gaussian), edges extended by half-sample reflection; sums in
 * double.  tmp: device scratch of n*nz*nx floats, aliasing neither in nor
 * out (in == out is allowed).  radius <= 127. */
int pyfwi_smooth(const float *in, float *out, float *tmp, int32_t n, int32_t nz, int32_t nx, const double *weights,
                 int32_t radius, void *stream);

/* Per-kernel timing.  While enabled, every step kernel the plan launches is
 * bracketed by CUDA events on the caller's stream.  pyfwi_profile_read
 * synchronises on those events and returns, for one kernel kind (0 forward
 * step, 1 adjoint+imaging step, 2 reverse step), the launches, the summed
 * device milliseconds and the summed grid cells x shots they processed; it
 * then clears the counters. */
int pyfwi_profile_enable(pyfwi_plan *plan, int32_t enable);
int pyfwi_profile_read(pyfwi_plan *plan, int32_t kind, int64_t *launches, double *ms, double *cell_shots);

/* Number of kernel tile variants the autotuner may choose between. */
int pyfwi_tile_count(int32_t half_order);

/* Kernel launches this plan issued since creation (for launch accounting). */
int pyfwi_launch_count(const pyfwi_plan *plan, int64_t *count);

/* What the plan made of the options that apply only where its layout
 * allows: *flags bit 0 persistent time loops (options.persist), bit 1
 * recompute beside the adjoint (options.overlap), bit 2 difference sets in the
 * checkpoint segments (options.store_diffs).  No reference counterpart. */
int pyfwi_plan_flags(const pyfwi_plan *plan, int32_t *flags);

/* Read and clear the workspace's device error word after the work queued on
 * `stream` (synchronises that stream).  *code: 0 none, 1 a streaming kernel
 * gave up waiting (one second) for a row copy and left its rows unwritten,
 * 2 a streaming kernel found its shared memory misaligned for copies, 3 a
 * persistent kernel gave up waiting (one second) at a grid barrier and left
 * its remaining steps undone.
 * Returns PYFWI_E_TIMEOUT when *code != 0.  The reference has no device-side
 * waits and no counterpart. */
int pyfwi_device_error(pyfwi_plan *plan, void *workspace, size_t bytes, int32_t *code, void *stream);

/* The forward states a reverse-mode plan keeps at its checkpoint steps, the
 * reference's WavePropagator.W (wave_propagation.py:150-156, filled at
 * :710-727): for shot s, checkpoint k and field f (vx, vz, taux, tauz,
 * tauxz), the state after internal step chp[k] on the padded grid.
 *   out  device [ns][nchp][5][nz+2npml][nx+2npml]
 * Valid after pyfwi_forward (pyfwi_gradient only reads the store).  Plans in
 * exact mode keep no such store: PYFWI_E_STATE.  Device-to-device copies on
 * `stream`; no kernel. */
int pyfwi_checkpoint_states(pyfwi_plan *plan, void *workspace, size_t bytes, float *out, void *stream);

/* Memory check (the GPU pool has no sanitizer): count the nonzero cells of
 * the zero frame around every FP32 plane of the workspace (materials, work
 * and adjoint states, gradient accumulators, checkpoint store) after the work
 * queued on `stream` (synchronises it).  The stencils read that frame as zero
 * and no kernel writes it, so *nonzero != 0 means a write outside the update
 * domain.  No reference counterpart. */
int pyfwi_frame_check(pyfwi_plan *plan, void *workspace, size_t bytes, int64_t *nonzero, void *stream);

/* Failure-path self test: one CTA waits on an mbarrier nothing arrives at,
 * with the streaming kernels' bounded wait cut to `limit_ns` (1e3 .. 1e10) of
 * the GPU's global timer, then gives up as they do and sets the workspace's
 * error word to 1.  Until pyfwi_device_error reads and clears the word, the
 * streaming kernels of later calls stop at once; the tile kernels run.  No
 * reference counterpart. */
int pyfwi_wait_selftest(pyfwi_plan *plan, void *workspace, size_t bytes, int64_t limit_ns, void *stream);

/* Failure-path self test of the persistent kernels' grid barrier: two CTAs
 * wait at the barrier for a third that does not exist, with the wait cut to
 * `limit_ns` (1e3 .. 1e10) of the GPU's global timer, then give up as a
 * persistent kernel does and set the workspace's error word to 3.  Until
 * pyfwi_device_error reads and clears the word, the persistent kernels of
 * later calls stop at their first barrier.  No reference counterpart. */
int pyfwi_barrier_selftest(pyfwi_plan *plan, void *workspace, size_t bytes, int64_t limit_ns, void *stream);

/* Gradient evaluation that allocates no device memory.  No counterpart in
 * the reference (PyFWI allocates its buffers through pyopencl per
 * WavePropagator).  For callers that cannot call cudaMalloc -- e.g. a host
 * program in another language with no CUDA allocator, or an application
 * whose memory pool owns the whole device -- this runs pyfwi_set_model,
 * pyfwi_forward, the L2 residual of every observed component and
 * pyfwi_gradient on one fixed array that the library holds in device memory
 * (PYFWI_STATIC_SCRATCH_BYTES on every GPU that loads it, until exit).
 *   vp .. src_vals, n_src   as pyfwi_set_model and pyfwi_forward
 *   observed  5 device pointers [nt_ext][ns*nr] of observed traces per raw
 *             component (vx, vz, taux, tauz, tauxz); NULL leaves a component
 *             out of the misfit
 *   grad      [3][nz][nx] as pyfwi_gradient;  misfit: device double, overwritten
 * Plans whose workspace + traces + residuals exceed the array are rejected
 * (PYFWI_E_WORKSPACE, message gives the bytes needed).  No call of this
 * entry point may be captured in a CUDA graph: the array is shared, so every
 * call rebuilds the plan's setup in it, including a copy of the source cells
 * from host memory.  The first call on a device looks up the array's device
 * address.  That address is kept until the process exits: after a
 * cudaDeviceReset of the device, do not call this entry point again in the
 * same process.  All calls on a device share the array (each call clears
 * what it needs); calls that overlap on the GPU race. */
#define PYFWI_STATIC_SCRATCH_BYTES (64u << 20)
int pyfwi_gradient_static(pyfwi_plan *plan, const float *vp, const float *vs, const float *rho,
                          const float *damp_x, const float *damp_z, const float *src_vals, int32_t n_src,
                          const float *const *observed, int32_t parameterization, float *grad, double *misfit,
                          void *stream);

const char *pyfwi_last_error(void);
int pyfwi_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PYFWI_B200_H */
