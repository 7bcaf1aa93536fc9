// Device code of the B200 elastic propagator.
//
// One kernel launch advances every shot of a batch by one time step.  Each
// CTA owns a TZ x TX tile of one shot (blockIdx.z) and fuses what the
// reference does in four to six full-grid OpenCL launches per step
// (PyFWI src/PyFWI/elastic.cl:155-308, 372-526, elastic_surface.cl:7-71):
//   forward  : source add -> velocity update on the tile plus an R-cell ring
//              -> stress update on the tile, reading the new velocities from
//              shared memory; receiver traces are recorded from the input
//              state (before the source add);
//   reverse  : the same with stress first (reverse-time reconstruction);
//   adjoint  : residual injection -> adjoint stress on tile + ring ->
//              adjoint velocity on the tile -> zero-lag imaging accumulation.
// Fields are FP32 planes in a padded layout (see Grid) whose frame is zero,
// so stencils never branch on the grid edge.  Arithmetic is FP32 with FMA.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pyfwi {

// Padded plane layout: grid cell (i, j) lives at (i + ZO) * pitch + (j + XO).
// The frame (ZO rows above/below, >= XO columns left/right) stays zero.
constexpr int XO = 8;
constexpr int ZO = 8;
constexpr int TX = 64;         // tile width in cells (all variants)
constexpr int NTHREADS = 256;  // threads per CTA (all variants)

enum Field { VX = 0, VZ = 1, TXX = 2, TZZ = 3, TXZ = 4 };

struct Grid {
    int tnz, tnx;    // padded grid (model + absorbing layer)
    int pitch;       // floats per allocated row, multiple of 32
    int rows;        // allocated rows, tnz + 2 * ZO
    long long plane; // pitch * rows
};

struct Coef {
    float cx[4];  // c_k / dh (x derivatives)
    float cz[4];  // c_k / dh (z derivatives)
    float dt;
};

struct Lines {
    int n;
    int row0[3], col0[3], drow[3], dcol[3], count[3], slot0[3], vzx[3];
};

__device__ __forceinline__ long long cell_off(const Grid &g, int i, int j)
{
    return (long long)(i + ZO) * g.pitch + (j + XO);
}

// One float4 of a padded plane; zero outside the allocation.  gj must be a
// multiple of 4 (rows start 128-byte aligned and XO is a multiple of 4).
__device__ __forceinline__ float4 ld4(const float *plane, const Grid &g, int gi, int gj)
{
    int ar = gi + ZO, ac = gj + XO;
    if (ar < 0 || ar >= g.rows || ac < 0 || ac + 3 >= g.pitch) return make_float4(0.f, 0.f, 0.f, 0.f);
    return __ldg(reinterpret_cast<const float4 *>(plane + (long long)ar * g.pitch + ac));
}

// ld4 through L2 only (ld.global.cg): for data other CTAs of the same
// launch wrote (the persistent kernels), which the read-only path may hold
// stale.
__device__ __forceinline__ float4 ld4c(const float *plane, const Grid &g, int gi, int gj)
{
    int ar = gi + ZO, ac = gj + XO;
    if (ar < 0 || ar >= g.rows || ac < 0 || ac + 3 >= g.pitch) return make_float4(0.f, 0.f, 0.f, 0.f);
    return __ldcg(reinterpret_cast<const float4 *>(plane + (long long)ar * g.pitch + ac));
}

__device__ __forceinline__ void st4s(float *s, float4 v) { *reinterpret_cast<float4 *>(s) = v; }

// Asynchronous 16-byte copy of the 4 cells (gi, gj .. gj+3) of `plane` into
// shared memory (cp.async, bypassing L1), zero-filled where ld4 reads zero.
__device__ __forceinline__ void cp4(float *dst, const float *plane, const Grid &g, int gi, int gj)
{
    const int ar = gi + ZO, ac = gj + XO;
    const bool ok = ar >= 0 && ar < g.rows && ac >= 0 && ac + 3 < g.pitch;
    const float *src = ok ? plane + (long long)ar * g.pitch + ac : plane;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(ok ? 16 : 0)
                 : "memory");
}

__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---- staggered one-sided differences on a shared-memory array -------------
// fwd: c1(f[+1]-f[0]) + c2(f[+2]-f[-1]) [+ c3(f[+3]-f[-2]) + c4(f[+4]-f[-3])]
// bwd: c1(f[0]-f[-1]) + c2(f[+1]-f[-2]) [+ c3(f[+2]-f[-3]) + c4(f[+3]-f[-4])]
// with c_k already divided by dh; s is the element stride of the direction.
template <int R>
__device__ __forceinline__ float dfwd(const float *f, int i, int s, const float *c)
{
    float r = c[0] * (f[i + s] - f[i]);
    r = fmaf(c[1], f[i + 2 * s] - f[i - s], r);
    if (R == 4) {
        r = fmaf(c[2], f[i + 3 * s] - f[i - 2 * s], r);
        r = fmaf(c[3], f[i + 4 * s] - f[i - 3 * s], r);
    }
    return r;
}

template <int R>
__device__ __forceinline__ float dbwd(const float *f, int i, int s, const float *c)
{
    float r = c[0] * (f[i] - f[i - s]);
    r = fmaf(c[1], f[i + s] - f[i - 2 * s], r);
    if (R == 4) {
        r = fmaf(c[2], f[i + 2 * s] - f[i - 3 * s], r);
        r = fmaf(c[3], f[i + 3 * s] - f[i - 4 * s], r);
    }
    return r;
}

// Differences of a pointwise product a*b (adjoint kernels, elastic.cl:385-463).
template <int R>
__device__ __forceinline__ float dfwd_p(const float *a, const float *b, int i, int s, const float *c)
{
#define P_(k) (a[(k)] * b[(k)])
    float r = c[0] * (P_(i + s) - P_(i));
    r = fmaf(c[1], P_(i + 2 * s) - P_(i - s), r);
    if (R == 4) {
        r = fmaf(c[2], P_(i + 3 * s) - P_(i - 2 * s), r);
        r = fmaf(c[3], P_(i + 4 * s) - P_(i - 3 * s), r);
    }
    return r;
}

template <int R>
__device__ __forceinline__ float dbwd_p(const float *a, const float *b, int i, int s, const float *c)
{
    float r = c[0] * (P_(i) - P_(i - s));
    r = fmaf(c[1], P_(i + s) - P_(i - 2 * s), r);
    if (R == 4) {
        r = fmaf(c[2], P_(i + 2 * s) - P_(i - 3 * s), r);
        r = fmaf(c[3], P_(i + 3 * s) - P_(i - 4 * s), r);
    }
    return r;
#undef P_
}

// Normal-stress pair of update_tauz (elastic.cl:235-270): txx gains
// dt ((lam + 2 mu) a + lam b), tzz gains dt (lam a + (lam + 2 mu) b), a = Dx+ vx,
// b = Dz- vz, then both are damped (forward, coeff = +1; the reverse step,
// coeff = -1, damps first and subtracts).  Every rounding is spelled out so
// that where mu = 0 (a fluid) the two increments are the same float: the
// fluid has no restoring force on txx - tzz, so a rounding difference between
// them (left to the compiler's choice of fused multiply-adds) would never
// radiate away and would grow step by step into the velocities.
__device__ __forceinline__ void normal_pair_fwd(float l, float m, float a, float b, float d, float dt, float &txx,
                                                float &tzz)
{
    const float l2m = l + 2.f * m;
    txx = __fmaf_rn(dt, __fmaf_rn(l2m, a, __fmul_rn(l, b)), txx);
    tzz = __fmaf_rn(dt, __fmaf_rn(l, a, __fmul_rn(l2m, b)), tzz);
    txx = __fmaf_rn(dt, __fmul_rn(-d, txx), txx);
    tzz = __fmaf_rn(dt, __fmul_rn(-d, tzz), tzz);
}

__device__ __forceinline__ void normal_pair_rev(float l, float m, float a, float b, float d, float dt, float &txx,
                                                float &tzz)
{
    const float l2m = l + 2.f * m;
    txx = __fmaf_rn(-dt, __fmul_rn(d, txx), txx);
    tzz = __fmaf_rn(-dt, __fmul_rn(d, tzz), tzz);
    txx = __fmaf_rn(-dt, __fmaf_rn(l2m, a, __fmul_rn(l, b)), txx);
    tzz = __fmaf_rn(-dt, __fmaf_rn(l, a, __fmul_rn(l2m, b)), tzz);
}

// Differences of (lam + 2 mu) * A.
template <int R>
__device__ __forceinline__ float dfwd_l2m(const float *lam, const float *mu, const float *A, int i, int s,
                                          const float *c)
{
#define L_(k) ((lam[(k)] + 2.f * mu[(k)]) * A[(k)])
    float r = c[0] * (L_(i + s) - L_(i));
    r = fmaf(c[1], L_(i + 2 * s) - L_(i - s), r);
    if (R == 4) {
        r = fmaf(c[2], L_(i + 3 * s) - L_(i - 2 * s), r);
        r = fmaf(c[3], L_(i + 4 * s) - L_(i - 3 * s), r);
    }
    return r;
}

template <int R>
__device__ __forceinline__ float dbwd_l2m(const float *lam, const float *mu, const float *A, int i, int s,
                                          const float *c)
{
    float r = c[0] * (L_(i) - L_(i - s));
    r = fmaf(c[1], L_(i + s) - L_(i - 2 * s), r);
    if (R == 4) {
        r = fmaf(c[2], L_(i + 2 * s) - L_(i - 3 * s), r);
        r = fmaf(c[3], L_(i + 3 * s) - L_(i - 4 * s), r);
    }
    return r;
#undef L_
}

// Same differences read straight from a global plane (imaging stencils).
template <int R>
__device__ __forceinline__ float gfwd(const float *f, long long i, long long s, const float *c)
{
    float r = c[0] * (__ldg(f + i + s) - __ldg(f + i));
    r = fmaf(c[1], __ldg(f + i + 2 * s) - __ldg(f + i - s), r);
    if (R == 4) {
        r = fmaf(c[2], __ldg(f + i + 3 * s) - __ldg(f + i - 2 * s), r);
        r = fmaf(c[3], __ldg(f + i + 4 * s) - __ldg(f + i - 3 * s), r);
    }
    return r;
}

template <int R>
__device__ __forceinline__ float gbwd(const float *f, long long i, long long s, const float *c)
{
    float r = c[0] * (__ldg(f + i) - __ldg(f + i - s));
    r = fmaf(c[1], __ldg(f + i + s) - __ldg(f + i - 2 * s), r);
    if (R == 4) {
        r = fmaf(c[2], __ldg(f + i + 2 * s) - __ldg(f + i - 3 * s), r);
        r = fmaf(c[3], __ldg(f + i + 3 * s) - __ldg(f + i - 4 * s), r);
    }
    return r;
}

// The same differences with the values taken through a loader ld(index):
// a snapshot plane widened to float, or an FP32 plane rounded to the
// snapshot format first (so that every forward state the exact adjoint
// reads from snapshots carries the same rounding, whichever slot holds it).

// 24-bit snapshots: the 24 leading bits of a float (sign, exponent, 15
// mantissa bits) rounded to nearest even, kept as a BF16 plane (the upper 16
// bits) and a byte plane (the next 8).  A BF16 snapshot is the same with no
// byte plane (rounded to its 16 bits instead).
__device__ __forceinline__ unsigned fp24_bits(float v)
{
    const unsigned u = __float_as_uint(v);
    return (u + 0x7Fu + ((u >> 8) & 1u)) >> 8;
}

__device__ __forceinline__ float fp24_round(float v) { return __uint_as_float(fp24_bits(v) << 8); }

// Snapshot value i: BF16 plane h, widened with byte plane l when l is set.
__device__ __forceinline__ float snapv(const __nv_bfloat16 *h, const unsigned char *l, long long i)
{
    const unsigned hi = reinterpret_cast<const unsigned short *>(h)[i];
    return __uint_as_float((hi << 16) | (l ? (unsigned)l[i] << 8 : 0u));
}

template <int R, typename L>
__device__ __forceinline__ float lfwd(L ld, long long i, long long s, const float *c)
{
    float r = c[0] * (ld(i + s) - ld(i));
    r = fmaf(c[1], ld(i + 2 * s) - ld(i - s), r);
    if (R == 4) {
        r = fmaf(c[2], ld(i + 3 * s) - ld(i - 2 * s), r);
        r = fmaf(c[3], ld(i + 4 * s) - ld(i - 3 * s), r);
    }
    return r;
}

template <int R, typename L>
__device__ __forceinline__ float lbwd(L ld, long long i, long long s, const float *c)
{
    float r = c[0] * (ld(i) - ld(i - s));
    r = fmaf(c[1], ld(i + s) - ld(i - 2 * s), r);
    if (R == 4) {
        r = fmaf(c[2], ld(i + 2 * s) - ld(i - 3 * s), r);
        r = fmaf(c[3], ld(i + 3 * s) - ld(i - 4 * s), r);
    }
    return r;
}

// Count the nonzero cells of the zero frame (rows outside [ZO, ZO + tnz),
// columns outside [XO, XO + tnx)) of n consecutive planes: the stencils rely
// on that frame reading as zero, and no kernel may write there.  NaN counts.
__global__ void frame_check_kernel(const float *base, long long nplanes, Grid g, unsigned long long *count)
{
    unsigned long long local = 0;
    const long long total = nplanes * g.plane;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long c = e % g.plane;
        const int i = (int)(c / g.pitch), j = (int)(c - (long long)i * g.pitch);
        const bool frame = i < ZO || i >= ZO + g.tnz || j < XO || j >= XO + g.tnx;
        if (frame && !(base[e] == 0.f)) ++local;
    }
    if (local) atomicAdd(count, local);
}

// ---------------------------------------------------------------------------
// kernel arguments
// ---------------------------------------------------------------------------
struct StepArgs {
    Grid g;
    Coef k;
    const float *in;       // input state of slot 0: [5][plane]
    float *out;            // output state of slot 0
    long long in_stride;   // elements between the states of consecutive slots
    long long out_stride;
    const float *mat;      // [4][plane]: lam, mu, buoyancy, rho
    const float *dampx;    // [pitch] damping per allocated column (x 1/s)
    const float *dampz;    // [rows] damping per allocated row
    int shot0;             // shot of slot 0
    const int *srcx;       // [ns] padded-grid source column per shot
    const int *srcz;       // [ns] source row per shot
    float4 src;            // (vx, vz, taux, tauz) added this step
    int add_src;
    int rec_row;           // trace row recorded this step, -1 for none
    float *traces;         // [5][nt_ext][ns*nr]
    long long trace_plane; // nt_ext * ns * nr
    int nr;
    int ns;
    Lines lines;
    int chunk;             // streaming kernels: grid rows per CTA
    __nv_bfloat16 *snap;   // nullable: BF16 copy of the output state, slot 0
    unsigned char *snap8;  // nullable: the byte planes of a 24-bit snapshot (snap holds the upper 16 bits)
    long long snap_stride; // elements between the snapshots of consecutive slots
    const float *tbase;    // streaming kernels: workspace base = row 0 of `tmap`
    int *err;              // streaming kernels: workspace error word
    // nullable: the imaging's differences of the output state (planes
    // Q_DXP_VX, Q_DZM_VZ, Q_VZS), and of the input state (planes Q_TXS,
    // Q_TZS), slot 0; written by fwd_step<R, TZ, QD>: FP32 planes (QD 1), or
    // BF16 planes of the upper 16 bits with byte planes qout8 / qin8 of the
    // next 8 (QD 2, 24-bit values)
    void *qout;
    void *qin;
    unsigned char *qout8, *qin8;
    long long q_stride;    // elements between the difference sets of consecutive slots
    int qlo, qhi_z, qhi_x; // the imaged cells: rows qlo .. qhi_z, columns qlo .. qhi_x (the only ones written)
    alignas(64) CUtensorMap tmap;  // streaming kernels: the workspace as rows of `pitch` floats
};

// The imaging's differences of a forward state S (elastic.cl:470-526), the
// five planes a difference set holds in place of S when the plan stores
// differences: what the zero-lag imaging of the adjoint step reads instead of
// differencing S itself.  The sums are those the imaging forms, in its order.
enum {
    Q_DXP_VX = 0,  // Dx+ vx
    Q_DZM_VZ = 1,  // Dz- vz
    Q_VZS = 2,     // Dz+ vz + Dx- vz  (the reference forms DzpVx from vz, elastic.cl:485)
    Q_TXS = 3,     // Dx- txx + Dz- txz
    Q_TZS = 4      // Dz+ tzz + Dx+ txz
};

// Snapshot of the five fields written at cell `co` (round to nearest even):
// BF16, or 24 bits when the byte planes sn8 are given.
__device__ __forceinline__ void write_snap1(__nv_bfloat16 *sn, unsigned char *sn8, long long o, float v)
{
    if (sn8) {
        const unsigned b = fp24_bits(v);
        sn[o] = __ushort_as_bfloat16((unsigned short)(b >> 8));
        sn8[o] = (unsigned char)(b & 0xFFu);
    } else {
        sn[o] = __float2bfloat16_rn(v);
    }
}

__device__ __forceinline__ void write_snap(__nv_bfloat16 *sn, unsigned char *sn8, long long P, long long co, float vx,
                                           float vz, float txx, float tzz, float txz)
{
    write_snap1(sn, sn8, VX * P + co, vx);
    write_snap1(sn, sn8, VZ * P + co, vz);
    write_snap1(sn, sn8, TXX * P + co, txx);
    write_snap1(sn, sn8, TZZ * P + co, tzz);
    write_snap1(sn, sn8, TXZ * P + co, txz);
}

struct AdjArgs {
    Grid g;
    Coef k;
    const float *in;       // adjoint state in, slot 0
    float *out;            // adjoint state out
    long long in_stride, out_stride;
    const float *fwd;      // forward state S_{t+1}, slot 0 (FP32)
    const __nv_bfloat16 *fwd16;  // same, BF16 snapshot (used when fwd == nullptr)
    const unsigned char *fwd8;   // nullable: byte planes of a 24-bit snapshot (with fwd16)
    long long fwd_stride;
    float *gacc;           // [slot][3 or 6][plane] accumulators
    long long gacc_stride;
    const float *mat;
    const float *dampx, *dampz;
    int npml;
    int shot0;
    int inj_row;           // residual row injected this step, -1 for none
    int epi_row;           // tile kernel: residual row the next step injects, added to this step's output (-1: none)
    const float *res[5];   // [nt_ext][ns*nr] residual components (nullable)
    int nr, ns;
    Lines lines;
    int chunk;             // streaming kernels: grid rows per CTA
    int nslots;            // tile kernel: shots in this launch (CTAs of blockIdx.z carry NS of them)
    const float *tbase;    // streaming kernels: workspace base = row 0 of `tmap`
    int *err;              // streaming kernels: workspace error word
    alignas(64) CUtensorMap tmap;  // streaming kernels: the workspace as rows of `pitch` floats
};

__device__ __forceinline__ bool in_domain(const Grid &g, int R, int i, int j)
{
    return i >= R && i <= g.tnz - R && j >= R && j <= g.tnx - R;
}

// Trace slot k of line l at cell (i, j), or -1 when no receiver of the line sits there.
__device__ __forceinline__ int line_slot(const Lines &L, int l, int i, int j)
{
    int d;
    if (L.drow[l] == 0) {
        d = j - L.col0[l];
        if (i != L.row0[l] || d < 0 || d % L.dcol[l]) return -1;
        d /= L.dcol[l];
    } else {
        d = i - L.row0[l];
        if (j != L.col0[l] || d < 0 || d % L.drow[l]) return -1;
        d /= L.drow[l];
    }
    return d < L.count[l] ? d : -1;
}

// Record the five fields of `st` at cell (i, j) into trace row `rec_row` of
// every trace slot whose receiver sits there.
__device__ __forceinline__ void record_cell(const StepArgs &a, int rec_row, const float *st, int shot, int i, int j)
{
    const Lines &L = a.lines;
    for (int l = 0; l < L.n; ++l) {
        int k;
        if (L.drow[l] == 0) {
            int d = j - L.col0[l];
            if (i != L.row0[l] || d < 0 || d % L.dcol[l]) continue;
            k = d / L.dcol[l];
        } else {
            int d = i - L.row0[l];
            if (j != L.col0[l] || d < 0 || d % L.drow[l]) continue;
            k = d / L.drow[l];
        }
        if (k >= L.count[l]) continue;
        long long o = (long long)rec_row * a.ns * a.nr + (long long)shot * a.nr + L.slot0[l] + k;
        long long c = cell_off(a.g, i, j);
        float vx = st[VX * a.g.plane + c];
        a.traces[0 * a.trace_plane + o] = vx;
        a.traces[1 * a.trace_plane + o] = L.vzx[l] ? vx : st[VZ * a.g.plane + c];
        a.traces[2 * a.trace_plane + o] = st[TXX * a.g.plane + c];
        a.traces[3 * a.trace_plane + o] = st[TZZ * a.g.plane + c];
        a.traces[4 * a.trace_plane + o] = st[TXZ * a.g.plane + c];
    }
}

// ---------------------------------------------------------------------------
// forward step: velocities then stresses (elastic.cl:155-308, coeff = +1)
// ---------------------------------------------------------------------------
template <int R, int TZ>
struct FwdShape {
    // Each thread updates 4 adjacent columns of one row from aligned float4
    // shared-memory loads, keeping the x-neighbours in registers.
    static constexpr int SW = TX + 16;     // stress row width: columns j0-8 .. j0+TX+7
    static constexpr int VW = TX + 8;      // velocity row width: columns j0-4 .. j0+TX+3
    static constexpr int HT = TZ + 4 * R;  // stress rows i0-2R ..
    static constexpr int HV = TZ + 2 * R;  // velocity rows i0-R ..
    static constexpr int FLOATS = 3 * HT * SW + 3 * HV * VW + 2 * TZ * TX;
    static_assert(R <= 4, "x halo of 4 columns per group");
};

__device__ __forceinline__ float4 ld4s(const float *s) { return *reinterpret_cast<const float4 *>(s); }
__device__ __forceinline__ float f4(const float4 &v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

// Difference planes: four values of one row from element o (a multiple of
// 4), or one value, as FP32 (QD 1) or 24 bits (QD 2: the upper 16 bits of
// the value rounded to nearest even at 15 mantissa bits in a BF16 plane q,
// the next 8 in a byte plane q8).
template <int QD>
__device__ __forceinline__ void qst4(void *q, unsigned char *q8, long long o, float4 v)
{
    if constexpr (QD == 1) {
        *reinterpret_cast<float4 *>(static_cast<float *>(q) + o) = v;
    } else {
        const unsigned b0 = fp24_bits(v.x), b1 = fp24_bits(v.y), b2 = fp24_bits(v.z), b3 = fp24_bits(v.w);
        *reinterpret_cast<uint2 *>(static_cast<__nv_bfloat16 *>(q) + o) =
            make_uint2((b0 >> 8) | ((b1 >> 8) << 16), (b2 >> 8) | ((b3 >> 8) << 16));
        *reinterpret_cast<unsigned *>(q8 + o) = (b0 & 0xFFu) | ((b1 & 0xFFu) << 8) | ((b2 & 0xFFu) << 16) | (b3 << 24);
    }
}

template <int QD>
__device__ __forceinline__ float qld(const float *F, const __nv_bfloat16 *F16, const unsigned char *F8, long long o)
{
    if constexpr (QD == 1) {
        return __ldg(F + o);
    } else {
        const unsigned hi = __ldg(reinterpret_cast<const unsigned short *>(F16) + o), lo = __ldg(F8 + o);
        return __uint_as_float((hi << 16) | (lo << 8));
    }
}

template <int QD>
__device__ __forceinline__ void qst1(void *q, unsigned char *q8, long long o, float v)
{
    if constexpr (QD == 1)
        static_cast<float *>(q)[o] = v;
    else
        write_snap1(static_cast<__nv_bfloat16 *>(q), q8, o, v);
}

// Three aligned float4 of a shared row around column c (c - 4 .. c + 7).
__device__ __forceinline__ void row12(float (&v)[12], const float *row, int c)
{
    const float4 a = ld4s(row + c - 4), b = ld4s(row + c), d = ld4s(row + c + 4);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    v[8] = d.x; v[9] = d.y; v[10] = d.z; v[11] = d.w;
}

// The differences of dfwd / dbwd, in the same operation order, on registers:
// x: v[4 + k] is column c + k; z: w[m] (float4 rows centre - R .. centre + R,
// w[R] the centre), component k.
template <int R>
__device__ __forceinline__ float xfwd(const float (&v)[12], int k, const float *c)
{
    const int o = 4 + k;
    float r = c[0] * (v[o + 1] - v[o]);
    r = fmaf(c[1], v[o + 2] - v[o - 1], r);
    if (R == 4) {
        r = fmaf(c[2], v[o + 3] - v[o - 2], r);
        r = fmaf(c[3], v[o + 4] - v[o - 3], r);
    }
    return r;
}

template <int R>
__device__ __forceinline__ float xbwd(const float (&v)[12], int k, const float *c)
{
    const int o = 4 + k;
    float r = c[0] * (v[o] - v[o - 1]);
    r = fmaf(c[1], v[o + 1] - v[o - 2], r);
    if (R == 4) {
        r = fmaf(c[2], v[o + 2] - v[o - 3], r);
        r = fmaf(c[3], v[o + 3] - v[o - 4], r);
    }
    return r;
}

template <int R>
__device__ __forceinline__ float zfwd(const float4 (&w)[2 * R + 1], int k, const float *c)
{
    float r = c[0] * (f4(w[R + 1], k) - f4(w[R], k));
    r = fmaf(c[1], f4(w[R + 2], k) - f4(w[R - 1], k), r);
    if (R == 4) {
        r = fmaf(c[2], f4(w[R + 3], k) - f4(w[R - 2], k), r);
        r = fmaf(c[3], f4(w[R + 4], k) - f4(w[R - 3], k), r);
    }
    return r;
}

template <int R>
__device__ __forceinline__ float zbwd(const float4 (&w)[2 * R + 1], int k, const float *c)
{
    float r = c[0] * (f4(w[R], k) - f4(w[R - 1], k));
    r = fmaf(c[1], f4(w[R + 1], k) - f4(w[R - 2], k), r);
    if (R == 4) {
        r = fmaf(c[2], f4(w[R + 2], k) - f4(w[R - 3], k), r);
        r = fmaf(c[3], f4(w[R + 3], k) - f4(w[R - 4], k), r);
    }
    return r;
}

// Rows centre - R .. centre + R of a shared plane at column c.
template <int R>
__device__ __forceinline__ void col_rows(float4 (&w)[2 * R + 1], const float *plane, int width, int centre, int c)
{
#pragma unroll
    for (int m = 0; m <= 2 * R; ++m) w[m] = ld4s(plane + (centre - R + m) * width + c);
}

// Damping of 4 columns from j (j a multiple of 4), zero outside the allocation.
__device__ __forceinline__ float4 damp4(const float *dampx, const Grid &g, int j)
{
    const int c = j + XO;
    if (c >= 0 && c + 3 < g.pitch) return __ldg(reinterpret_cast<const float4 *>(dampx + c));
    float4 v;
    v.x = (c >= 0 && c < g.pitch) ? __ldg(dampx + c) : 0.f;
    v.y = (c + 1 >= 0 && c + 1 < g.pitch) ? __ldg(dampx + c + 1) : 0.f;
    v.z = (c + 2 >= 0 && c + 2 < g.pitch) ? __ldg(dampx + c + 2) : 0.f;
    v.w = (c + 3 >= 0 && c + 3 < g.pitch) ? __ldg(dampx + c + 3) : 0.f;
    return v;
}

// What changes from one forward step to the next: the input and output
// states (slot 0 and the element stride between slots), the source sample
// and the trace row recorded (-1: none), the snapshot planes written.
// StepArgs has the same fields: the step kernel passes its arguments
// themselves (read from parameter space where they are used).
struct StepVar {
    const float *in;
    float *out;
    long long in_stride, out_stride;
    float4 src;
    int add_src;
    int rec_row;
    __nv_bfloat16 *snap;
    unsigned char *snap8;
};

// One forward step of tile (bx, by) of slot `slot`; sm: FwdShape::FLOATS
// floats of shared memory.  Ends with shared memory still in use: a caller
// that reuses it for another tile synchronises first.
// W24: snapshots are written as 24 bits (sv.snap8 set), else as BF16.
// STAGED: the caller has put the tile's input in shared memory already (the
// TMA kernel); otherwise it is copied here with cp.async.
template <int R, int TZ, bool W24, class V, bool STAGED = false>
__device__ __forceinline__ void fwd_tile(const StepArgs &a, const V &sv, int bx, int by, int slot, float *sm)
{
    using S = FwdShape<R, TZ>;
    constexpr int SW = S::SW, VW = S::VW, HT = S::HT, HV = S::HV;
    float *s_txx = sm, *s_tzz = s_txx + HT * SW, *s_txz = s_tzz + HT * SW;
    float *s_vx = s_txz + HT * SW, *s_vz = s_vx + HV * VW, *s_b = s_vz + HV * VW;
    float *s_lam = s_b + HV * VW, *s_mu = s_lam + TZ * TX;  // the tile's cells

    const Grid &g = a.g;
    const long long P = g.plane;
    const int shot = a.shot0 + slot;
    const int j0 = bx * TX, i0 = by * TZ;
    const float *in = sv.in + slot * sv.in_stride;
    float *out = sv.out + slot * sv.out_stride;
    const int tid = threadIdx.x;
    const float dt = a.k.dt;

    // every copy of the tile in flight at once, then one wait
    for (int e = tid; !STAGED && e < HT * (SW / 4); e += NTHREADS) {
        int r = e / (SW / 4), q = e - r * (SW / 4);
        int gi = i0 - 2 * R + r, gj = j0 - 8 + 4 * q, o = r * SW + 4 * q;
        cp4(s_txx + o, in + TXX * P, g, gi, gj);
        cp4(s_tzz + o, in + TZZ * P, g, gi, gj);
        cp4(s_txz + o, in + TXZ * P, g, gi, gj);
    }
    for (int e = tid; !STAGED && e < HV * (VW / 4); e += NTHREADS) {
        int r = e / (VW / 4), q = e - r * (VW / 4);
        int gi = i0 - R + r, gj = j0 - 4 + 4 * q, o = r * VW + 4 * q;
        cp4(s_vx + o, in + VX * P, g, gi, gj);
        cp4(s_vz + o, in + VZ * P, g, gi, gj);
        cp4(s_b + o, a.mat + 2 * P, g, gi, gj);
    }
    for (int e = tid; !STAGED && e < TZ * (TX / 4); e += NTHREADS) {
        int r = e / (TX / 4), q = e - r * (TX / 4), o = r * TX + 4 * q;
        cp4(s_lam + o, a.mat, g, i0 + r, j0 + 4 * q);
        cp4(s_mu + o, a.mat + P, g, i0 + r, j0 + 4 * q);
    }
    if (!STAGED) {
        cp_wait_all();
        __syncthreads();
    }
    if (sv.add_src && tid == 0) {  // wave_propagation.py:652-664, elastic_surface.cl:23-28
        const int si = a.srcz[shot], sj = a.srcx[shot];
        const int ct = sj - (j0 - 8), cv = sj - (j0 - 4), rt = si - (i0 - 2 * R), rv = si - (i0 - R);
        if (ct >= 0 && ct < SW && rt >= 0 && rt < HT) {
            s_txx[rt * SW + ct] += sv.src.z;
            s_tzz[rt * SW + ct] += sv.src.w;
        }
        if (cv >= 0 && cv < VW && rv >= 0 && rv < HV) {
            s_vx[rv * VW + cv] += sv.src.x;
            s_vz[rv * VW + cv] += sv.src.y;
        }
    }
    __syncthreads();

    // velocities (update_velx / update_velz) on rows i0-R .. and columns
    // j0-4 .., 4 columns per thread
    for (int e = tid; e < HV * (VW / 4); e += NTHREADS) {
        const int r = e / (VW / 4), q = e - r * (VW / 4);
        const int gi = i0 - R + r, gj = j0 - 4 + 4 * q;
        const int rt = r + R, ct = 4 * q + 4, o = r * VW + 4 * q;
        float4 vx = ld4s(s_vx + o), vz = ld4s(s_vz + o);
        const float4 b = ld4s(s_b + o), dx = damp4(a.dampx, g, gj);
        const float dz = (gi + ZO >= 0 && gi + ZO < g.rows) ? __ldg(a.dampz + gi + ZO) : 0.f;
        float t[12];
        float4 w[2 * R + 1];
        float rx[4], rz[4];
        row12(t, s_txx + rt * SW, ct);  // Dx- txx
#pragma unroll
        for (int k = 0; k < 4; ++k) rx[k] = xbwd<R>(t, k, a.k.cx);
        col_rows<R>(w, s_txz, SW, rt, ct);  // Dz- txz
#pragma unroll
        for (int k = 0; k < 4; ++k) rz[k] = zbwd<R>(w, k, a.k.cz);
        float nvx[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float v = f4(vx, k);
            if (in_domain(g, R, gi, gj + k)) {
                const float d = f4(dx, k) + dz;
                v = v + dt * (f4(b, k) * (rx[k] + rz[k]));
                v = v + dt * (-d * v);
            }
            nvx[k] = v;
        }
        row12(t, s_txz + rt * SW, ct);  // Dx+ txz
#pragma unroll
        for (int k = 0; k < 4; ++k) rx[k] = xfwd<R>(t, k, a.k.cx);
        col_rows<R>(w, s_tzz, SW, rt, ct);  // Dz+ tzz
#pragma unroll
        for (int k = 0; k < 4; ++k) rz[k] = zfwd<R>(w, k, a.k.cz);
        float nvz[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float v = f4(vz, k);
            if (in_domain(g, R, gi, gj + k)) {
                const float d = f4(dx, k) + dz;
                v = v + dt * (f4(b, k) * (rz[k] + rx[k]));
                v = v + dt * (-d * v);
            }
            nvz[k] = v;
        }
        st4s(s_vx + o, make_float4(nvx[0], nvx[1], nvx[2], nvx[3]));
        st4s(s_vz + o, make_float4(nvz[0], nvz[1], nvz[2], nvz[3]));
    }
    __syncthreads();

    // stresses (update_tauz / update_tauxz) on the tile, 4 columns per thread
    for (int e = tid; e < TZ * (TX / 4); e += NTHREADS) {
        const int r = e / (TX / 4), q = e - r * (TX / 4);
        const int gi = i0 + r, gj = j0 + 4 * q;
        if (gi >= g.tnz || gj >= g.tnx) continue;
        const int rv = r + R, cv = 4 * q + 4, rt = r + 2 * R, ct = 4 * q + 8;
        const long long co = cell_off(g, gi, gj);
        const float4 vxc = ld4s(s_vx + rv * VW + cv), vzc = ld4s(s_vz + rv * VW + cv);
        float4 txx = ld4s(s_txx + rt * SW + ct), tzz = ld4s(s_tzz + rt * SW + ct), txz = ld4s(s_txz + rt * SW + ct);
        const float4 lam = ld4s(s_lam + r * TX + 4 * q), mu = ld4s(s_mu + r * TX + 4 * q),
                     dx = damp4(a.dampx, g, gj);
        const float dz = __ldg(a.dampz + gi + ZO);
        float t[12];
        float4 w[2 * R + 1];
        float dxp_vx[4], dzm_vz[4], dxm_vz[4], dzp_vx[4];
        row12(t, s_vx + rv * VW, cv);
#pragma unroll
        for (int k = 0; k < 4; ++k) dxp_vx[k] = xfwd<R>(t, k, a.k.cx);
        row12(t, s_vz + rv * VW, cv);
#pragma unroll
        for (int k = 0; k < 4; ++k) dxm_vz[k] = xbwd<R>(t, k, a.k.cx);
        col_rows<R>(w, s_vz, VW, rv, cv);
#pragma unroll
        for (int k = 0; k < 4; ++k) dzm_vz[k] = zbwd<R>(w, k, a.k.cz);
        col_rows<R>(w, s_vx, VW, rv, cv);
#pragma unroll
        for (int k = 0; k < 4; ++k) dzp_vx[k] = zfwd<R>(w, k, a.k.cz);
        float oxx[4], ozz[4], oxz[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float sxx = f4(txx, k), szz = f4(tzz, k), sxz = f4(txz, k);
            if (in_domain(g, R, gi, gj + k)) {
                const float l = f4(lam, k), m = f4(mu, k), d = f4(dx, k) + dz;
                normal_pair_fwd(l, m, dxp_vx[k], dzm_vz[k], d, dt, sxx, szz);
                sxz = sxz + dt * (m * (dxm_vz[k] + dzp_vx[k]));
                sxz = sxz + dt * (-d * sxz);
            }
            oxx[k] = sxx;
            ozz[k] = szz;
            oxz[k] = sxz;
        }
        if (gj + 3 < g.tnx) {
            *reinterpret_cast<float4 *>(out + VX * P + co) = vxc;
            *reinterpret_cast<float4 *>(out + VZ * P + co) = vzc;
            *reinterpret_cast<float4 *>(out + TXX * P + co) = make_float4(oxx[0], oxx[1], oxx[2], oxx[3]);
            *reinterpret_cast<float4 *>(out + TZZ * P + co) = make_float4(ozz[0], ozz[1], ozz[2], ozz[3]);
            *reinterpret_cast<float4 *>(out + TXZ * P + co) = make_float4(oxz[0], oxz[1], oxz[2], oxz[3]);
        } else {
            for (int k = 0; k < 4 && gj + k < g.tnx; ++k) {
                out[VX * P + co + k] = f4(vxc, k);
                out[VZ * P + co + k] = f4(vzc, k);
                out[TXX * P + co + k] = oxx[k];
                out[TZZ * P + co + k] = ozz[k];
                out[TXZ * P + co + k] = oxz[k];
            }
        }
        for (int k = 0; k < 4 && gj + k < g.tnx; ++k) {
            if (sv.snap)
                write_snap(sv.snap + slot * a.snap_stride, W24 ? sv.snap8 + slot * a.snap_stride : nullptr, P,
                           co + k, f4(vxc, k), f4(vzc, k), oxx[k], ozz[k], oxz[k]);
            if (sv.rec_row >= 0) record_cell(a, sv.rec_row, in, shot, gi, gj + k);
        }
    }
}

// The step kernels.  fwd_step24 writes 24-bit snapshots through fwd_tile.
// fwd_step (every other forward step) keeps its own copy of the tile code:
// measured on B200 the same code reached through fwd_tile ran 3 % slower on
// the 64-shot survey (the compiler allocates the two differently), so the
// shared tile function serves the 24-bit, TMA-staged and persistent forms.
template <int R, int TZ>
__global__ void __launch_bounds__(NTHREADS) fwd_step24(const __grid_constant__ StepArgs a)
{
    extern __shared__ float4 smem4[];
    fwd_tile<R, TZ, true>(a, a, blockIdx.x, blockIdx.y, blockIdx.z, reinterpret_cast<float *>(smem4));
}

// QD (1: FP32, 2: 24 bits): the step also writes the imaging's differences
// of its output state (a.qout: velocity planes) and of its input state
// (a.qin, nullable: stress planes) for the adjoint to read in place of the
// stored state; four more floats of shared memory (the input stresses at the
// source cell before this step's source is added), at most 64 registers
// (4 CTAs per SM) at half order 2.
template <int R, int TZ, int QD = 0>
__global__ void __launch_bounds__(NTHREADS, QD ? (R == 2 ? 4 : 2) : 0) fwd_step(const __grid_constant__ StepArgs a)
{
    using S = FwdShape<R, TZ>;
    constexpr int SW = S::SW, VW = S::VW, HT = S::HT, HV = S::HV;
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4);
    float *s_txx = sm, *s_tzz = s_txx + HT * SW, *s_txz = s_tzz + HT * SW;
    float *s_vx = s_txz + HT * SW, *s_vz = s_vx + HV * VW, *s_b = s_vz + HV * VW;
    float *s_lam = s_b + HV * VW, *s_mu = s_lam + TZ * TX;  // the tile's cells

    const Grid &g = a.g;
    const long long P = g.plane;
    const int slot = blockIdx.z, shot = a.shot0 + slot;
    const int j0 = blockIdx.x * TX, i0 = blockIdx.y * TZ;
    const float *in = a.in + slot * a.in_stride;
    float *out = a.out + slot * a.out_stride;
    const int tid = threadIdx.x;
    const float dt = a.k.dt;

    // the source cell, read while the tile's copies are in flight
    int src_i = 0, src_j = 0;
    if (a.add_src && tid == 0) {
        src_i = __ldg(a.srcz + shot);
        src_j = __ldg(a.srcx + shot);
    }
    // every copy of the tile in flight at once, then one wait
    for (int e = tid; e < HT * (SW / 4); e += NTHREADS) {
        int r = e / (SW / 4), q = e - r * (SW / 4);
        int gi = i0 - 2 * R + r, gj = j0 - 8 + 4 * q, o = r * SW + 4 * q;
        cp4(s_txx + o, in + TXX * P, g, gi, gj);
        cp4(s_tzz + o, in + TZZ * P, g, gi, gj);
        cp4(s_txz + o, in + TXZ * P, g, gi, gj);
    }
    for (int e = tid; e < HV * (VW / 4); e += NTHREADS) {
        int r = e / (VW / 4), q = e - r * (VW / 4);
        int gi = i0 - R + r, gj = j0 - 4 + 4 * q, o = r * VW + 4 * q;
        cp4(s_vx + o, in + VX * P, g, gi, gj);
        cp4(s_vz + o, in + VZ * P, g, gi, gj);
        cp4(s_b + o, a.mat + 2 * P, g, gi, gj);
    }
    for (int e = tid; e < TZ * (TX / 4); e += NTHREADS) {
        int r = e / (TX / 4), q = e - r * (TX / 4), o = r * TX + 4 * q;
        cp4(s_lam + o, a.mat, g, i0 + r, j0 + 4 * q);
        cp4(s_mu + o, a.mat + P, g, i0 + r, j0 + 4 * q);
    }
    cp_wait_all();
    __syncthreads();
    if (a.add_src) {  // wave_propagation.py:652-664, elastic_surface.cl:23-28 (uniform: a barrier only then)
        if (tid == 0) {
            const int si = src_i, sj = src_j;
            const int ct = sj - (j0 - 8), cv = sj - (j0 - 4), rt = si - (i0 - 2 * R), rv = si - (i0 - R);
            if (ct >= 0 && ct < SW && rt >= 0 && rt < HT) {
                if constexpr (QD) {  // the stored input state has no source of this step
                    s_mu[TZ * TX] = s_txx[rt * SW + ct];
                    s_mu[TZ * TX + 1] = s_tzz[rt * SW + ct];
                }
                s_txx[rt * SW + ct] += a.src.z;
                s_tzz[rt * SW + ct] += a.src.w;
            }
            if (cv >= 0 && cv < VW && rv >= 0 && rv < HV) {
                s_vx[rv * VW + cv] += a.src.x;
                s_vz[rv * VW + cv] += a.src.y;
            }
        }
        __syncthreads();
    }

    // velocities (update_velx / update_velz) on rows i0-R .. and columns
    // j0-4 .., 4 columns per thread
    for (int e = tid; e < HV * (VW / 4); e += NTHREADS) {
        const int r = e / (VW / 4), q = e - r * (VW / 4);
        const int gi = i0 - R + r, gj = j0 - 4 + 4 * q;
        const int rt = r + R, ct = 4 * q + 4, o = r * VW + 4 * q;
        float4 vx = ld4s(s_vx + o), vz = ld4s(s_vz + o);
        const float4 b = ld4s(s_b + o), dx = damp4(a.dampx, g, gj);
        const float dz = (gi + ZO >= 0 && gi + ZO < g.rows) ? __ldg(a.dampz + gi + ZO) : 0.f;
        float t[12];
        float4 w[2 * R + 1];
        float rx[4], rz[4];
        row12(t, s_txx + rt * SW, ct);  // Dx- txx
#pragma unroll
        for (int k = 0; k < 4; ++k) rx[k] = xbwd<R>(t, k, a.k.cx);
        col_rows<R>(w, s_txz, SW, rt, ct);  // Dz- txz
#pragma unroll
        for (int k = 0; k < 4; ++k) rz[k] = zbwd<R>(w, k, a.k.cz);
        float nvx[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float v = f4(vx, k);
            if (in_domain(g, R, gi, gj + k)) {
                const float d = f4(dx, k) + dz;
                v = v + dt * (f4(b, k) * (rx[k] + rz[k]));
                v = v + dt * (-d * v);
            }
            nvx[k] = v;
        }
        const bool qtile = QD && a.qin && r >= R && r < R + TZ && q >= 1 && q <= TX / 4 && gi >= a.qlo &&
                           gi <= a.qhi_z && gj + 3 >= a.qlo && gj <= a.qhi_x;
        if constexpr (QD) {
            if (qtile)
                qst4<QD>(a.qin, a.qin8, slot * a.q_stride + Q_TXS * P + cell_off(g, gi, gj),
                         make_float4(rx[0] + rz[0], rx[1] + rz[1], rx[2] + rz[2], rx[3] + rz[3]));
        }
        row12(t, s_txz + rt * SW, ct);  // Dx+ txz
#pragma unroll
        for (int k = 0; k < 4; ++k) rx[k] = xfwd<R>(t, k, a.k.cx);
        col_rows<R>(w, s_tzz, SW, rt, ct);  // Dz+ tzz
#pragma unroll
        for (int k = 0; k < 4; ++k) rz[k] = zfwd<R>(w, k, a.k.cz);
        float nvz[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float v = f4(vz, k);
            if (in_domain(g, R, gi, gj + k)) {
                const float d = f4(dx, k) + dz;
                v = v + dt * (f4(b, k) * (rz[k] + rx[k]));
                v = v + dt * (-d * v);
            }
            nvz[k] = v;
        }
        if constexpr (QD) {
            if (qtile)
                qst4<QD>(a.qin, a.qin8, slot * a.q_stride + Q_TZS * P + cell_off(g, gi, gj),
                         make_float4(rz[0] + rx[0], rz[1] + rx[1], rz[2] + rx[2], rz[3] + rx[3]));
        }
        st4s(s_vx + o, make_float4(nvx[0], nvx[1], nvx[2], nvx[3]));
        st4s(s_vz + o, make_float4(nvz[0], nvz[1], nvz[2], nvz[3]));
    }
    __syncthreads();
    if constexpr (QD) {
        // The stress differences above saw this step's source at its cell;
        // the imaging wants those of the stored input state: thread 0
        // recomputes the cells whose stencils reach the source cell (row si,
        // columns sj-R+1 .. sj+R for Dx- txx; column sj, rows si-R .. si+R-1
        // for Dz+ tzz) with the values from before the source was added, and
        // overwrites them (ordered after the loop's stores by the barrier).
        if (a.qin && a.add_src && tid == 0) {
            const int si = a.srcz[shot], sj = a.srcx[shot];
            const int rt = si - (i0 - 2 * R), ct = sj - (j0 - 8);
            if (ct >= 0 && ct < SW && rt >= 0 && rt < HT) {
                const long long src = (long long)rt * SW + ct;
                const float oxx = s_mu[TZ * TX], ozz = s_mu[TZ * TX + 1];
                auto lxx = [&](long long k) { return k == src ? oxx : s_txx[k]; };
                auto lzz = [&](long long k) { return k == src ? ozz : s_tzz[k]; };
                auto lxz = [&](long long k) { return s_txz[k]; };
                const long long qo = slot * a.q_stride;
                for (int m = 0; m < 4 * R; ++m) {
                    const int gi = m < 2 * R ? si : si - R + (m - 2 * R);
                    const int gj = m < 2 * R ? sj - R + 1 + m : sj;
                    if (gi < i0 || gi >= i0 + TZ || gj < j0 || gj >= j0 + TX || gi >= g.tnz || gj >= g.tnx) continue;
                    const long long c = (long long)(gi - (i0 - 2 * R)) * SW + (gj - (j0 - 8));
                    const long long co = cell_off(g, gi, gj);
                    qst1<QD>(a.qin, a.qin8, qo + Q_TXS * P + co, lbwd<R>(lxx, c, 1, a.k.cx) + lbwd<R>(lxz, c, SW, a.k.cz));
                    qst1<QD>(a.qin, a.qin8, qo + Q_TZS * P + co, lfwd<R>(lzz, c, SW, a.k.cz) + lfwd<R>(lxz, c, 1, a.k.cx));
                }
            }
        }
    }

    // stresses (update_tauz / update_tauxz) on the tile, 4 columns per thread
    for (int e = tid; e < TZ * (TX / 4); e += NTHREADS) {
        const int r = e / (TX / 4), q = e - r * (TX / 4);
        const int gi = i0 + r, gj = j0 + 4 * q;
        if (gi >= g.tnz || gj >= g.tnx) continue;
        const int rv = r + R, cv = 4 * q + 4, rt = r + 2 * R, ct = 4 * q + 8;
        const long long co = cell_off(g, gi, gj);
        const float4 vxc = ld4s(s_vx + rv * VW + cv), vzc = ld4s(s_vz + rv * VW + cv);
        float4 txx = ld4s(s_txx + rt * SW + ct), tzz = ld4s(s_tzz + rt * SW + ct), txz = ld4s(s_txz + rt * SW + ct);
        const float4 lam = ld4s(s_lam + r * TX + 4 * q), mu = ld4s(s_mu + r * TX + 4 * q),
                     dx = damp4(a.dampx, g, gj);
        const float dz = __ldg(a.dampz + gi + ZO);
        float t[12];
        float4 w[2 * R + 1];
        float dxp_vx[4], dzm_vz[4], dxm_vz[4], dzp_vx[4];
        row12(t, s_vx + rv * VW, cv);
#pragma unroll
        for (int k = 0; k < 4; ++k) dxp_vx[k] = xfwd<R>(t, k, a.k.cx);
        row12(t, s_vz + rv * VW, cv);
#pragma unroll
        for (int k = 0; k < 4; ++k) dxm_vz[k] = xbwd<R>(t, k, a.k.cx);
        if constexpr (QD) {  // Dz+ vz + Dx- vz of the output state, from scalar shared loads
            if (a.qout && gi >= a.qlo && gi <= a.qhi_z && gj + 3 >= a.qlo && gj <= a.qhi_x) {
                const int iv = rv * VW + cv;
                qst4<QD>(a.qout, a.qout8, slot * a.q_stride + Q_VZS * P + co,
                     make_float4(dfwd<R>(s_vz, iv, VW, a.k.cz) + dxm_vz[0], dfwd<R>(s_vz, iv + 1, VW, a.k.cz) + dxm_vz[1],
                                 dfwd<R>(s_vz, iv + 2, VW, a.k.cz) + dxm_vz[2],
                                 dfwd<R>(s_vz, iv + 3, VW, a.k.cz) + dxm_vz[3]));
            }
        }
        col_rows<R>(w, s_vz, VW, rv, cv);
#pragma unroll
        for (int k = 0; k < 4; ++k) dzm_vz[k] = zbwd<R>(w, k, a.k.cz);
        col_rows<R>(w, s_vx, VW, rv, cv);
#pragma unroll
        for (int k = 0; k < 4; ++k) dzp_vx[k] = zfwd<R>(w, k, a.k.cz);
        float oxx[4], ozz[4], oxz[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float sxx = f4(txx, k), szz = f4(tzz, k), sxz = f4(txz, k);
            if (in_domain(g, R, gi, gj + k)) {
                const float l = f4(lam, k), m = f4(mu, k), d = f4(dx, k) + dz;
                normal_pair_fwd(l, m, dxp_vx[k], dzm_vz[k], d, dt, sxx, szz);
                sxz = sxz + dt * (m * (dxm_vz[k] + dzp_vx[k]));
                sxz = sxz + dt * (-d * sxz);
            }
            oxx[k] = sxx;
            ozz[k] = szz;
            oxz[k] = sxz;
        }
        if constexpr (QD) {  // the velocity differences of the output state
            if (a.qout && gi >= a.qlo && gi <= a.qhi_z && gj + 3 >= a.qlo && gj <= a.qhi_x) {
                const long long qo = slot * a.q_stride + co;
                qst4<QD>(a.qout, a.qout8, qo + Q_DXP_VX * P, make_float4(dxp_vx[0], dxp_vx[1], dxp_vx[2], dxp_vx[3]));
                qst4<QD>(a.qout, a.qout8, qo + Q_DZM_VZ * P, make_float4(dzm_vz[0], dzm_vz[1], dzm_vz[2], dzm_vz[3]));
            }
        }
        if (gj + 3 < g.tnx) {
            *reinterpret_cast<float4 *>(out + VX * P + co) = vxc;
            *reinterpret_cast<float4 *>(out + VZ * P + co) = vzc;
            *reinterpret_cast<float4 *>(out + TXX * P + co) = make_float4(oxx[0], oxx[1], oxx[2], oxx[3]);
            *reinterpret_cast<float4 *>(out + TZZ * P + co) = make_float4(ozz[0], ozz[1], ozz[2], ozz[3]);
            *reinterpret_cast<float4 *>(out + TXZ * P + co) = make_float4(oxz[0], oxz[1], oxz[2], oxz[3]);
        } else {
            for (int k = 0; k < 4 && gj + k < g.tnx; ++k) {
                out[VX * P + co + k] = f4(vxc, k);
                out[VZ * P + co + k] = f4(vzc, k);
                out[TXX * P + co + k] = oxx[k];
                out[TZZ * P + co + k] = ozz[k];
                out[TXZ * P + co + k] = oxz[k];
            }
        }
        for (int k = 0; k < 4 && gj + k < g.tnx; ++k) {
            if (a.snap)
                write_snap(a.snap + slot * a.snap_stride, nullptr, P, co + k, f4(vxc, k), f4(vzc, k), oxx[k], ozz[k], oxz[k]);
            if (a.rec_row >= 0) record_cell(a, a.rec_row, in, shot, gi, gj + k);
        }
    }
}

// ---------------------------------------------------------------------------
// reverse-time step: stresses then velocities, coeff = -1 (elastic.cl:175-306,
// order of wave_propagation.py:782-812).  Used only by the reference's
// chpr < 100 checkpoint scheme.
// ---------------------------------------------------------------------------
template <int R, int TZ>
struct RevShape {
    static constexpr int W = TX + 4 * R;
    static constexpr int HT = TZ + 4 * R;  // velocity rows
    static constexpr int HV = TZ + 2 * R;  // stress rows
    static constexpr int FLOATS = 2 * HT * W + 5 * HV * W;
};

template <int R, int TZ>
__global__ void __launch_bounds__(NTHREADS) rev_step(const __grid_constant__ StepArgs a)
{
    using S = RevShape<R, TZ>;
    constexpr int W = S::W, HT = S::HT, HV = S::HV, VW = TX + 2 * R;
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4);
    float *s_vx = sm, *s_vz = s_vx + HT * W;
    float *s_txx = s_vz + HT * W, *s_tzz = s_txx + HV * W, *s_txz = s_tzz + HV * W;
    float *s_lam = s_txz + HV * W, *s_mu = s_lam + HV * W;

    const Grid &g = a.g;
    const int slot = blockIdx.z;
    const int j0 = blockIdx.x * TX, i0 = blockIdx.y * TZ, sx0 = j0 - 2 * R;
    const float *in = a.in + slot * a.in_stride;
    float *out = a.out + slot * a.out_stride;
    const int tid = threadIdx.x;
    const float dt = a.k.dt;

    for (int e = tid; e < HT * (W / 4); e += NTHREADS) {
        int r = e / (W / 4), q = e - r * (W / 4);
        int gi = i0 - 2 * R + r, gj = sx0 + 4 * q, o = r * W + 4 * q;
        st4s(s_vx + o, ld4(in + VX * g.plane, g, gi, gj));
        st4s(s_vz + o, ld4(in + VZ * g.plane, g, gi, gj));
    }
    for (int e = tid; e < HV * (W / 4); e += NTHREADS) {
        int r = e / (W / 4), q = e - r * (W / 4);
        int gi = i0 - R + r, gj = sx0 + 4 * q, o = r * W + 4 * q;
        st4s(s_txx + o, ld4(in + TXX * g.plane, g, gi, gj));
        st4s(s_tzz + o, ld4(in + TZZ * g.plane, g, gi, gj));
        st4s(s_txz + o, ld4(in + TXZ * g.plane, g, gi, gj));
        st4s(s_lam + o, ld4(a.mat, g, gi, gj));
        st4s(s_mu + o, ld4(a.mat + g.plane, g, gi, gj));
    }
    __syncthreads();

    for (int e = tid; e < HV * VW; e += NTHREADS) {
        int r = e / VW, cc = e - r * VW;
        int gi = i0 - R + r, gj = j0 - R + cc;
        if (!in_domain(g, R, gi, gj)) continue;
        int is = r * W + cc + R, iv = is + R * W;
        float d = __ldg(a.dampx + gj + XO) + __ldg(a.dampz + gi + ZO);
        float lam = s_lam[is], mu = s_mu[is];
        float dxp_vx = dfwd<R>(s_vx, iv, 1, a.k.cx), dzm_vz = dbwd<R>(s_vz, iv, W, a.k.cz);
        float dxm_vz = dbwd<R>(s_vz, iv, 1, a.k.cx), dzp_vx = dfwd<R>(s_vx, iv, W, a.k.cz);
        float txz = s_txz[is];
        txz = txz - dt * (d * txz);
        txz = txz - dt * (mu * (dxm_vz + dzp_vx));
        float txx = s_txx[is], tzz = s_tzz[is];
        normal_pair_rev(lam, mu, dxp_vx, dzm_vz, d, dt, txx, tzz);
        s_txx[is] = txx;
        s_tzz[is] = tzz;
        s_txz[is] = txz;
    }
    __syncthreads();

    const int c = tid % TX;
    const int gj = j0 + c;
    if (gj >= g.tnx) return;
    for (int r = tid / TX; r < TZ; r += NTHREADS / TX) {
        int gi = i0 + r;
        if (gi >= g.tnz) break;
        int is = (r + R) * W + c + 2 * R, iv = is + R * W;
        float vx = s_vx[iv], vz = s_vz[iv];
        long long co = cell_off(g, gi, gj);
        if (in_domain(g, R, gi, gj)) {
            float b = __ldg(a.mat + 2 * g.plane + co);
            float d = __ldg(a.dampx + gj + XO) + __ldg(a.dampz + gi + ZO);
            vz = vz - dt * (d * vz);
            vz = vz - dt * (b * (dfwd<R>(s_tzz, is, W, a.k.cz) + dfwd<R>(s_txz, is, 1, a.k.cx)));
            vx = vx - dt * (d * vx);
            vx = vx - dt * (b * (dbwd<R>(s_txx, is, 1, a.k.cx) + dbwd<R>(s_txz, is, W, a.k.cz)));
        }
        out[VX * g.plane + co] = vx;
        out[VZ * g.plane + co] = vz;
        out[TXX * g.plane + co] = s_txx[is];
        out[TZZ * g.plane + co] = s_tzz[is];
        out[TXZ * g.plane + co] = s_txz[is];
    }
}

// ---------------------------------------------------------------------------
// adjoint step + imaging (Adj_injSrc, Adj_update_tau, Adj_update_v, Grad:
// elastic_surface.cl:48-71, elastic.cl:316-526)
// ---------------------------------------------------------------------------
// Differences along a register window w[0..2R] (w[R] is the centre row).
template <int R, int N>
__device__ __forceinline__ float wfwd(const float (&w)[N], const float *c)
{
    float r = c[0] * (w[R + 1] - w[R]);
    r = fmaf(c[1], w[R + 2] - w[R - 1], r);
    if (R == 4) {
        r = fmaf(c[2], w[R + 3] - w[R - 2], r);
        r = fmaf(c[3], w[R + 4] - w[R - 3], r);
    }
    return r;
}

template <int R, int N>
__device__ __forceinline__ float wbwd(const float (&w)[N], const float *c)
{
    float r = c[0] * (w[R] - w[R - 1]);
    r = fmaf(c[1], w[R + 1] - w[R - 2], r);
    if (R == 4) {
        r = fmaf(c[2], w[R + 2] - w[R - 3], r);
        r = fmaf(c[3], w[R + 3] - w[R - 4], r);
    }
    return r;
}

template <int N>
__device__ __forceinline__ void shift(float (&w)[N], float top)
{
#pragma unroll
    for (int q = 0; q < N - 1; ++q) w[q] = w[q + 1];
    w[N - 1] = top;
}

template <int R, int TZ>
struct AdjShape {
    static constexpr int W = TX + 4 * R;
    static constexpr int HT = TZ + 4 * R;  // b * adjoint velocity rows
    static constexpr int HV = TZ + 2 * R;  // adjoint stress rows
    static constexpr int FLOATS = 2 * HT * W + 3 * HV * W;
};


// The next step's residual row epi_row added at cell (i, j) of
// the output: to the adjoint velocities in registers and the stresses in
// memory, one receiver line after another.
__device__ __forceinline__ void inject_epilogue(const AdjArgs &a, int epi_row, int slot, int i, int j, long long co, float &avx,
                                                float &avz, float *out)
{
    const long long P = a.g.plane;
    for (int l = 0; l < a.lines.n; ++l) {
        const int ks = line_slot(a.lines, l, i, j);
        if (ks < 0) continue;
        const long long o = (long long)epi_row * a.ns * a.nr + (long long)(a.shot0 + slot) * a.nr + a.lines.slot0[l] + ks;
        if (a.res[0]) avx += __ldg(a.res[0] + o);
        if (a.res[1]) avz += __ldg(a.res[1] + o);
        for (int f = TXX; f <= TXZ; ++f)
            if (a.res[f]) out[f * P + co] += __ldg(a.res[f] + o);
    }
}

// CTAs per SM the adjoint step is built for (the register bound of its
// launch): 6 with one shot per CTA (40 registers, 31 KB of shared memory),
// 5 when each CTA carries NS > 1 shots (their summed accumulators take
// another 12 KB of shared memory).
template <int R, bool ENERGY, int NS>
struct AdjOccupancy {
    static constexpr int value = (R == 2 && !ENERGY) ? (NS == 1 ? 6 : NS == 2 ? 5 : 4) : 1;
};

// Shared-memory floats of the adjoint step: the staged fields, plus the
// CTA's accumulators when it carries several shots.
template <int R, int TZ, bool ENERGY, int NS>
constexpr int adj_smem_floats()
{
    return AdjShape<R, TZ>::FLOATS + (NS > 1 ? (ENERGY ? 6 : 3) * TZ * TX : 0);
}

// One adjoint step of NS shots per CTA (blockIdx.z covers slots
// blockIdx.z * NS ..): the shots of a CTA run one after another over the
// same tile and add their imaging into accumulator slot blockIdx.z.  With
// NS > 1 the accumulators of the tile's cells stay in shared memory across
// the shots (each thread owns its cells' entries) and are read and written
// in global memory once, instead of once per shot; the sums run in shot
// order, then over slots in the final reduction.
// What changes from one adjoint step to the next: the input and output
// adjoint states, the forward state S(t+1) the imaging reads (FP32, or a
// BF16 / 24-bit snapshot), and the residual row the next step injects.
// AdjArgs has the same fields: the step kernel passes its arguments
// themselves.
struct AdjVar {
    const float *in;
    float *out;
    const float *fwd;
    const __nv_bfloat16 *fwd16;
    const unsigned char *fwd8;
    int epi_row;
};

// One adjoint step of tile (bx, by) for the slots bz * NS ..; sm:
// adj_smem_floats floats of shared memory.  Ends with shared memory still in
// use: a caller that reuses it for another tile synchronises first.
// COH: the input adjoint state and the accumulators are read through L2
// (written by other CTAs of the same launch: the persistent kernel).
template <int R, int TZ, bool ENERGY, int NS, bool NARROW, bool COH, class V>
__device__ __forceinline__ void adj_tile(const AdjArgs &a, const V &av, int bx, int by, int bz, float *sm)
{
    using S = AdjShape<R, TZ>;
    constexpr int W = S::W, HT = S::HT, HV = S::HV, VW = TX + 2 * R;
    constexpr int NACC = ENERGY ? 6 : 3;
    // rows i0-2R ..: b*Avx and b*Avz (the operands of the adjoint stress
    // differences); after the stress update they hold lam*Atx and
    // (lam+2mu)*Atz on rows i0-R ..
    float *s_pvx = sm, *s_pvz = s_pvx + HT * W;
    // rows i0-R ..: Atx, Atz, Atxz; after the stress update (lam+2mu)*Atx,
    // lam*Atz, mu*Atxz (the operands of the adjoint velocity differences)
    float *s_atx = s_pvz + HT * W, *s_atz = s_atx + HV * W, *s_atxz = s_atz + HV * W;

    const Grid &g = a.g;
    const long long P = g.plane;
    const int j0 = bx * TX, i0 = by * TZ, sx0 = j0 - 2 * R;
    const int tid = threadIdx.x;
    const float dt = a.k.dt;

    // adjoint velocities and imaging: each thread takes NK consecutive rows
    // of one column, so the z differences of the imaging slide down register
    // windows (rows gi-R .. gi+R of the forward vz, tzz and txz): one new
    // row per field and cell
    constexpr int NK = TZ / (NTHREADS / TX);
    const int c = tid % TX;
    const int gj = j0 + c;
    const int r0 = (tid / TX) * NK;
    const int glo = a.npml + R;
    const bool col_img = gj >= glo && gj <= g.tnx - R - a.npml;  // this column is imaged (Grad's domain)
    float *G = a.gacc + bz * a.gacc_stride;
    // NS > 1: the CTA's shots summed in shared memory, [NACC][TZ][TX]
    float *s_acc = s_atxz + HV * W;
    if (NS > 1) {
        for (int k = 0; k < NK; ++k) {
            const int gi = i0 + r0 + k;
            const bool im = col_img && gi >= glo && gi <= g.tnz - R - a.npml;
            const long long co = im ? cell_off(g, gi, gj) : 0;
#pragma unroll
            for (int f = 0; f < NACC; ++f) s_acc[(f * TZ + r0 + k) * TX + c] = im ? G[f * P + co] : 0.f;
        }
    }

    for (int q = 0; q < NS; ++q) {
        const int slot = bz * NS + q;
        if (slot >= a.nslots) break;  // the same for every thread of the CTA
        if (q) __syncthreads();       // the previous shot is done with shared memory
        const float *in = av.in + slot * a.in_stride;
        float *out = av.out + slot * a.out_stride;

        // the stresses as asynchronous copies, in flight while the velocity
        // products are loaded and stored
        for (int e = tid; e < HV * (W / 4); e += NTHREADS) {
            int r = e / (W / 4), q = e - r * (W / 4);
            int gi = i0 - R + r, gj = sx0 + 4 * q, o = r * W + 4 * q;
            cp4(s_atx + o, in + TXX * P, g, gi, gj);
            cp4(s_atz + o, in + TZZ * P, g, gi, gj);
            cp4(s_atxz + o, in + TXZ * P, g, gi, gj);
        }
        for (int e = tid; e < HT * (W / 4); e += NTHREADS) {
            int r = e / (W / 4), q = e - r * (W / 4);
            int gi = i0 - 2 * R + r, gj = sx0 + 4 * q, o = r * W + 4 * q;
            const float4 b = ld4(a.mat + 2 * P, g, gi, gj);
            const float4 vx = COH ? ld4c(in + VX * P, g, gi, gj) : ld4(in + VX * P, g, gi, gj);
            const float4 vz = COH ? ld4c(in + VZ * P, g, gi, gj) : ld4(in + VZ * P, g, gi, gj);
            st4s(s_pvx + o, make_float4(vx.x * b.x, vx.y * b.y, vx.z * b.z, vx.w * b.w));
            st4s(s_pvz + o, make_float4(vz.x * b.x, vz.y * b.y, vz.z * b.z, vz.w * b.w));
        }
        cp_wait_all();
        __syncthreads();

        // adjoint stresses on the tile plus an R-cell ring (Adj_update_tau); the
        // tile's own cells go straight to the output
        for (int e = tid; e < HV * VW; e += NTHREADS) {
            int r = e / VW, cc = e - r * VW;
            int gi = i0 - R + r, gj = j0 - R + cc;
            int is = r * W + cc + R, iv = is + R * W;
            const bool tile = r >= R && r < R + TZ && cc >= R && cc < R + TX && gi < g.tnz && gj < g.tnx;
            float atx = s_atx[is], atz = s_atz[is], atxz = s_atxz[is];
            if (in_domain(g, R, gi, gj)) {
                float dx = __ldg(a.dampx + gj + XO), dz = __ldg(a.dampz + gi + ZO);
                atx = atx + (-dt) * (dx * atx + dfwd<R>(s_pvx, iv, 1, a.k.cx));
                atz = atz + (-dt) * (dz * atz + dbwd<R>(s_pvz, iv, W, a.k.cz));
                atxz = atxz + (-dt) * ((dx + dz) * atxz + (dfwd<R>(s_pvx, iv, W, a.k.cz) + dbwd<R>(s_pvz, iv, 1, a.k.cx)));
                s_atx[is] = atx;
                s_atz[is] = atz;
                s_atxz[is] = atxz;
            }
            if (tile) {
                const long long co = cell_off(g, gi, gj);
                out[TXX * P + co] = atx;
                out[TZZ * P + co] = atz;
                out[TXZ * P + co] = atxz;
            }
        }
        __syncthreads();

        // material products of the new adjoint stresses
        for (int e = tid; e < HV * VW; e += NTHREADS) {
            int r = e / VW, cc = e - r * VW;
            int gi = i0 - R + r, gj = j0 - R + cc;
            int is = r * W + cc + R;
            // lam = mu = 0 in the zero frame and beyond the allocated rows / columns
            const bool alloc = gi + ZO >= 0 && gi + ZO < g.rows && gj + XO >= 0 && gj + XO < g.pitch;
            const long long co = alloc ? cell_off(g, gi, gj) : 0;
            const float lam = alloc ? __ldg(a.mat + co) : 0.f, mu = alloc ? __ldg(a.mat + P + co) : 0.f;
            const float l2m = lam + 2.f * mu;
            const float atx = s_atx[is], atz = s_atz[is], atxz = s_atxz[is];
            s_atx[is] = l2m * atx;
            s_atz[is] = lam * atz;
            s_atxz[is] = mu * atxz;
            s_pvx[is] = lam * atx;
            s_pvz[is] = l2m * atz;
        }
        __syncthreads();

        // adjoint velocities on the tile (Adj_update_v) and imaging (Grad)
        if (gj >= g.tnx) continue;
        // the imaged forward state: FP32, or (NARROW) BF16 / 24-bit snapshots
        const float *F = !NARROW && av.fwd ? av.fwd + slot * a.fwd_stride : nullptr;
        const __nv_bfloat16 *F16 = NARROW ? av.fwd16 + slot * a.fwd_stride : nullptr;
        const unsigned char *F8 = NARROW && av.fwd8 ? av.fwd8 + slot * a.fwd_stride : nullptr;
        const long long pz = g.pitch;
        float wvz[2 * R + 1], wtz[2 * R + 1], wtxz[2 * R + 1];
        const bool win = !NARROW && F && col_img && i0 + r0 + NK - 1 >= glo && i0 + r0 <= g.tnz - R - a.npml;
        if (win) {
            const long long c0 = cell_off(g, i0 + r0, gj);
#pragma unroll
            for (int m = 0; m < 2 * R; ++m) {
                const long long o = c0 + (m - R) * pz;
                wvz[m + 1] = __ldg(F + VZ * P + o);
                wtz[m + 1] = __ldg(F + TZZ * P + o);
                wtxz[m + 1] = __ldg(F + TXZ * P + o);
            }
        }
        for (int k = 0; k < NK; ++k) {
            const int r = r0 + k, gi = i0 + r;
            if (gi >= g.tnz) break;
            int is = (r + R) * W + c + 2 * R;
            long long co = cell_off(g, gi, gj);
            if (win) {  // the window moves to rows gi-R .. gi+R
                const long long o = co + R * pz;
                shift(wvz, __ldg(F + VZ * P + o));
                shift(wtz, __ldg(F + TZZ * P + o));
                shift(wtxz, __ldg(F + TXZ * P + o));
            }
            float avx = COH ? __ldcg(in + VX * P + co) : __ldg(in + VX * P + co);
            float avz = COH ? __ldcg(in + VZ * P + co) : __ldg(in + VZ * P + co);
            if (in_domain(g, R, gi, gj)) {
                float dx = __ldg(a.dampx + gj + XO), dz = __ldg(a.dampz + gi + ZO);
                float sx = dbwd<R>(s_atx, is, 1, a.k.cx) + dbwd<R>(s_atz, is, 1, a.k.cx) + dbwd<R>(s_atxz, is, W, a.k.cz);
                float sz = dfwd<R>(s_pvx, is, W, a.k.cz) + dfwd<R>(s_pvz, is, W, a.k.cz) + dfwd<R>(s_atxz, is, 1, a.k.cx);
                avx = avx + (-dt) * ((2.f * dx + dz) * avx + sx);
                avz = avz + (-dt) * ((dx + 2.f * dz) * avz + sz);
            }
            if (col_img && gi >= glo && gi <= g.tnz - R - a.npml) {
                const long long sz_ = g.pitch;
                // the new adjoint stresses this CTA wrote above (plain loads: written in this kernel)
                const float atx = out[TXX * P + co], atz = out[TZZ * P + co], atxz = out[TXZ * P + co];
                float dzp_vx, dxm_vz, dxp_vx, dzm_vz, dzp_tz, dxm_tx, dxp_txz, dzm_txz;
                float vx = 0.f, vz = 0.f, tx = 0.f, tz = 0.f, txz = 0.f;
                if (!NARROW) {
                    // DzpVx is formed from vz, as the reference does (elastic.cl:485)
                    dzp_vx = wfwd<R>(wvz, a.k.cz);
                    dxm_vz = gbwd<R>(F + VZ * P, co, 1, a.k.cx);
                    dxp_vx = gfwd<R>(F + VX * P, co, 1, a.k.cx);
                    dzm_vz = wbwd<R>(wvz, a.k.cz);
                    dzp_tz = wfwd<R>(wtz, a.k.cz);
                    dxm_tx = gbwd<R>(F + TXX * P, co, 1, a.k.cx);
                    dxp_txz = gfwd<R>(F + TXZ * P, co, 1, a.k.cx);
                    dzm_txz = wbwd<R>(wtxz, a.k.cz);
                    if (ENERGY) {
                        vx = F[VX * P + co];
                        vz = wvz[R];
                        tx = F[TXX * P + co];
                        tz = wtz[R];
                        txz = wtxz[R];
                    }
                } else {
#define B16F(f, k) snapv(F16, F8, (f) * P + (k))
#define BFWD(f, s)                                                                                       \
    (a.k.c##s[0] * (B16F(f, co + st) - B16F(f, co)) + a.k.c##s[1] * (B16F(f, co + 2 * st) - B16F(f, co - st)) + \
     (R == 4 ? a.k.c##s[2] * (B16F(f, co + 3 * st) - B16F(f, co - 2 * st)) +                              \
                   a.k.c##s[3] * (B16F(f, co + 4 * st) - B16F(f, co - 3 * st))                            \
             : 0.f))
#define BBWD(f, s)                                                                                       \
    (a.k.c##s[0] * (B16F(f, co) - B16F(f, co - st)) + a.k.c##s[1] * (B16F(f, co + st) - B16F(f, co - 2 * st)) + \
     (R == 4 ? a.k.c##s[2] * (B16F(f, co + 2 * st) - B16F(f, co - 3 * st)) +                              \
                   a.k.c##s[3] * (B16F(f, co + 3 * st) - B16F(f, co - 4 * st))                            \
             : 0.f))
                    long long st = sz_;
                    dzp_vx = BFWD(VZ, z);
                    dzm_vz = BBWD(VZ, z);
                    dzp_tz = BFWD(TZZ, z);
                    dzm_txz = BBWD(TXZ, z);
                    st = 1;
                    dxm_vz = BBWD(VZ, x);
                    dxp_vx = BFWD(VX, x);
                    dxm_tx = BBWD(TXX, x);
                    dxp_txz = BFWD(TXZ, x);
                    if (ENERGY) {
                        vx = B16F(VX, co);
                        vz = B16F(VZ, co);
                        tx = B16F(TXX, co);
                        tz = B16F(TZZ, co);
                        txz = B16F(TXZ, co);
                    }
#undef B16F
#undef BFWD
#undef BBWD
                }
                const float b = __ldg(a.mat + 2 * P + co);
                float img[NACC];
                if (NS == 1) {  // one shot: read-modify-write in memory, as each step of the reference's Grad
#pragma unroll
                    for (int f = 0; f < NACC; ++f) img[f] = COH ? __ldcg(G + f * P + co) : G[f * P + co];
                } else {
#pragma unroll
                    for (int f = 0; f < NACC; ++f) img[f] = s_acc[(f * TZ + r) * TX + c];
                }
                img[0] += 2.f * dt * (atx * dxp_vx + atz * dzm_vz) + dt * atxz * (dzp_vx + dxm_vz);
                img[1] += dt * (atx + atz) * (dxp_vx + dzm_vz);
                img[2] += -(dt * (b * b)) * (avx * (dxm_tx + dzm_txz) + avz * (dzp_tz + dxp_txz));
                if (ENERGY) {
                    float dt2 = dt * dt;
                    img[3 % NACC] += 4.f * dt2 * (tx * tx * dxp_vx * dxp_vx + tz * tz * dzm_vz * dzm_vz) +
                                     dt2 * txz * txz * (dzp_vx * dzp_vx + dxm_vz * dxm_vz);
                    img[4 % NACC] += dt2 * (tx * tx + tz * tz) * (dxp_vx * dxp_vx + dzm_vz * dzm_vz);
                    img[5 % NACC] += dt2 * (vx * vx * (dxm_tx * dxm_tx + dzm_txz * dzm_txz) +
                                            vz * vz * (dzp_tz * dzp_tz + dxp_txz * dxp_txz));
                }
                if (NS == 1) {
#pragma unroll
                    for (int f = 0; f < NACC; ++f) G[f * P + co] = img[f];
                } else {
#pragma unroll
                    for (int f = 0; f < NACC; ++f) s_acc[(f * TZ + r) * TX + c] = img[f];
                }
            }
            // the residual the next step injects (Adj_injSrc, elastic_surface.cl:48-71),
            // added to this step's output after the imaging has read it
            if (av.epi_row >= 0) inject_epilogue(a, av.epi_row, slot, gi, gj, co, avx, avz, out);
            out[VX * P + co] = avx;
            out[VZ * P + co] = avz;
        }
    }
    if (NS > 1) {
        for (int k = 0; k < NK; ++k) {
            const int gi = i0 + r0 + k;
            if (col_img && gi >= glo && gi <= g.tnz - R - a.npml) {
                const long long co = cell_off(g, gi, gj);
#pragma unroll
                for (int f = 0; f < NACC; ++f) G[f * P + co] = s_acc[(f * TZ + r0 + k) * TX + c];
            }
        }
    }
}

// The adjoint step kernels through adj_tile: NS shots per CTA, and (NARROW)
// the imaging reading BF16 or 24-bit snapshots (fwd16, fwd8) instead of FP32
// states.
template <int R, int TZ, bool ENERGY, int NS, bool NARROW>
__global__ void __launch_bounds__(NTHREADS, AdjOccupancy<R, ENERGY, NS>::value)
    adj_step_ns(const __grid_constant__ AdjArgs a)
{
    extern __shared__ float4 smem4[];
    adj_tile<R, TZ, ENERGY, NS, NARROW, false>(a, a, blockIdx.x, blockIdx.y, blockIdx.z,
                                               reinterpret_cast<float *>(smem4));
}

__device__ __forceinline__ float bf(const __nv_bfloat16 *p, long long i) { return __bfloat162float(p[i]); }

// adj_step: one shot per CTA, FP32 or BF16 imaged states (the default), with
// its own copy of the tile code: measured on B200 the same code reached
// through adj_tile ran 5 % slower on the 64-shot survey.
// PF (variant 11, no energy terms): the tile's three gradient accumulators
// are copied into shared memory by cp.async at the start, in flight with the
// stress copies, so the imaging's read-modify-write no longer waits on them
// in global memory (12 KB more shared memory: 5 CTAs per SM).
// QD (no energy terms): a.fwd is the difference set of S_{t+1} (planes
// Q_*), written by the forward step, so the imaging reads five values per
// cell instead of differencing the stored state.  (Without the difference
// windows it fits 32 registers and 7 CTAs per SM, measured slower on B200
// than 6: 0.96 against 0.83 ms per 64-shot launch.)
template <int R, int TZ, bool ENERGY, bool PF = false, int QD = 0>
__global__ void __launch_bounds__(NTHREADS, (R == 2 && !ENERGY) ? (PF ? 5 : 6) : 1)
    adj_step(const __grid_constant__ AdjArgs a)
{
    using S = AdjShape<R, TZ>;
    constexpr int W = S::W, HT = S::HT, HV = S::HV, VW = TX + 2 * R;
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4);
    // rows i0-2R ..: b*Avx and b*Avz (the operands of the adjoint stress
    // differences); after the stress update they hold lam*Atx and
    // (lam+2mu)*Atz on rows i0-R ..
    float *s_pvx = sm, *s_pvz = s_pvx + HT * W;
    // rows i0-R ..: Atx, Atz, Atxz; after the stress update (lam+2mu)*Atx,
    // lam*Atz, mu*Atxz (the operands of the adjoint velocity differences)
    float *s_atx = s_pvz + HT * W, *s_atz = s_atx + HV * W, *s_atxz = s_atz + HV * W;

    const Grid &g = a.g;
    const long long P = g.plane;
    const int slot = blockIdx.z;
    const int j0 = blockIdx.x * TX, i0 = blockIdx.y * TZ, sx0 = j0 - 2 * R;
    const float *in = a.in + slot * a.in_stride;
    float *out = a.out + slot * a.out_stride;
    const int tid = threadIdx.x;
    const float dt = a.k.dt;
    float *s_g = s_atxz + HV * W;  // PF: [3][TZ][TX] the tile's accumulators

    if (PF) {  // the accumulators first: their copies wait the longest (DRAM)
        const float *Gs = a.gacc + slot * a.gacc_stride;
        for (int e = tid; e < 3 * TZ * (TX / 4); e += NTHREADS) {
            const int f = e / (TZ * (TX / 4)), rem = e - f * (TZ * (TX / 4)), r = rem / (TX / 4), q = rem - r * (TX / 4);
            cp4(s_g + (f * TZ + r) * TX + 4 * q, Gs + f * P, g, i0 + r, j0 + 4 * q);
        }
    }
    // the stresses as asynchronous copies, in flight while the velocity
    // products are loaded and stored
    for (int e = tid; e < HV * (W / 4); e += NTHREADS) {
        int r = e / (W / 4), q = e - r * (W / 4);
        int gi = i0 - R + r, gj = sx0 + 4 * q, o = r * W + 4 * q;
        cp4(s_atx + o, in + TXX * P, g, gi, gj);
        cp4(s_atz + o, in + TZZ * P, g, gi, gj);
        cp4(s_atxz + o, in + TXZ * P, g, gi, gj);
    }
    for (int e = tid; e < HT * (W / 4); e += NTHREADS) {
        int r = e / (W / 4), q = e - r * (W / 4);
        int gi = i0 - 2 * R + r, gj = sx0 + 4 * q, o = r * W + 4 * q;
        const float4 b = ld4(a.mat + 2 * P, g, gi, gj), vx = ld4(in + VX * P, g, gi, gj),
                     vz = ld4(in + VZ * P, g, gi, gj);
        st4s(s_pvx + o, make_float4(vx.x * b.x, vx.y * b.y, vx.z * b.z, vx.w * b.w));
        st4s(s_pvz + o, make_float4(vz.x * b.x, vz.y * b.y, vz.z * b.z, vz.w * b.w));
    }
    cp_wait_all();
    __syncthreads();

    // adjoint stresses on the tile plus an R-cell ring (Adj_update_tau); the
    // tile's own cells go straight to the output
    for (int e = tid; e < HV * VW; e += NTHREADS) {
        int r = e / VW, cc = e - r * VW;
        int gi = i0 - R + r, gj = j0 - R + cc;
        int is = r * W + cc + R, iv = is + R * W;
        const bool tile = r >= R && r < R + TZ && cc >= R && cc < R + TX && gi < g.tnz && gj < g.tnx;
        float atx = s_atx[is], atz = s_atz[is], atxz = s_atxz[is];
        if (in_domain(g, R, gi, gj)) {
            float dx = __ldg(a.dampx + gj + XO), dz = __ldg(a.dampz + gi + ZO);
            atx = atx + (-dt) * (dx * atx + dfwd<R>(s_pvx, iv, 1, a.k.cx));
            atz = atz + (-dt) * (dz * atz + dbwd<R>(s_pvz, iv, W, a.k.cz));
            atxz = atxz + (-dt) * ((dx + dz) * atxz + (dfwd<R>(s_pvx, iv, W, a.k.cz) + dbwd<R>(s_pvz, iv, 1, a.k.cx)));
            s_atx[is] = atx;
            s_atz[is] = atz;
            s_atxz[is] = atxz;
        }
        if (tile) {
            const long long co = cell_off(g, gi, gj);
            out[TXX * P + co] = atx;
            out[TZZ * P + co] = atz;
            out[TXZ * P + co] = atxz;
        }
    }
    __syncthreads();

    // material products of the new adjoint stresses
    for (int e = tid; e < HV * VW; e += NTHREADS) {
        int r = e / VW, cc = e - r * VW;
        int gi = i0 - R + r, gj = j0 - R + cc;
        int is = r * W + cc + R;
        // lam = mu = 0 in the zero frame and beyond the allocated rows / columns
        const bool alloc = gi + ZO >= 0 && gi + ZO < g.rows && gj + XO >= 0 && gj + XO < g.pitch;
        const long long co = alloc ? cell_off(g, gi, gj) : 0;
        const float lam = alloc ? __ldg(a.mat + co) : 0.f, mu = alloc ? __ldg(a.mat + P + co) : 0.f;
        const float l2m = lam + 2.f * mu;
        const float atx = s_atx[is], atz = s_atz[is], atxz = s_atxz[is];
        s_atx[is] = l2m * atx;
        s_atz[is] = lam * atz;
        s_atxz[is] = mu * atxz;
        s_pvx[is] = lam * atx;
        s_pvz[is] = l2m * atz;
    }
    __syncthreads();

    // adjoint velocities on the tile (Adj_update_v) and imaging (Grad)
    const int c = tid % TX;
    const int gj = j0 + c;
    if (gj >= g.tnx) return;
    const int glo = a.npml + R;
    const float *F = a.fwd ? a.fwd + slot * a.fwd_stride : nullptr;
    const __nv_bfloat16 *F16 = a.fwd16 ? a.fwd16 + slot * a.fwd_stride : nullptr;
    float *G = a.gacc + slot * a.gacc_stride;
    // each thread takes NK consecutive rows of its column, so the z
    // differences of the imaging slide down register windows (rows gi-R ..
    // gi+R of the forward vz, tzz and txz): one new row per field and cell
    constexpr int NK = TZ / (NTHREADS / TX);
    const int r0 = (tid / TX) * NK;
    const long long pz = g.pitch;
    float wvz[2 * R + 1], wtz[2 * R + 1], wtxz[2 * R + 1];
    const bool win = QD == 0 && F && gj >= glo && gj <= g.tnx - R - a.npml && i0 + r0 + NK - 1 >= glo &&
                     i0 + r0 <= g.tnz - R - a.npml;
    if (win) {
        const long long c0 = cell_off(g, i0 + r0, gj);
#pragma unroll
        for (int m = 0; m < 2 * R; ++m) {
            const long long o = c0 + (m - R) * pz;
            wvz[m + 1] = __ldg(F + VZ * P + o);
            wtz[m + 1] = __ldg(F + TZZ * P + o);
            wtxz[m + 1] = __ldg(F + TXZ * P + o);
        }
    }
    for (int k = 0; k < NK; ++k) {
        const int r = r0 + k, gi = i0 + r;
        if (gi >= g.tnz) break;
        int is = (r + R) * W + c + 2 * R;
        long long co = cell_off(g, gi, gj);
        if (win) {  // the window moves to rows gi-R .. gi+R
            const long long o = co + R * pz;
            shift(wvz, __ldg(F + VZ * P + o));
            shift(wtz, __ldg(F + TZZ * P + o));
            shift(wtxz, __ldg(F + TXZ * P + o));
        }
        float avx = __ldg(in + VX * P + co), avz = __ldg(in + VZ * P + co);
        if (in_domain(g, R, gi, gj)) {
            float dx = __ldg(a.dampx + gj + XO), dz = __ldg(a.dampz + gi + ZO);
            float sx = dbwd<R>(s_atx, is, 1, a.k.cx) + dbwd<R>(s_atz, is, 1, a.k.cx) + dbwd<R>(s_atxz, is, W, a.k.cz);
            float sz = dfwd<R>(s_pvx, is, W, a.k.cz) + dfwd<R>(s_pvz, is, W, a.k.cz) + dfwd<R>(s_atxz, is, 1, a.k.cx);
            avx = avx + (-dt) * ((2.f * dx + dz) * avx + sx);
            avz = avz + (-dt) * ((dx + 2.f * dz) * avz + sz);
        }
        if (!(gi < glo || gi > g.tnz - R - a.npml || gj < glo || gj > g.tnx - R - a.npml)) {
        const long long sz_ = g.pitch;
        // the new adjoint stresses this CTA wrote above (plain loads: written in this kernel)
        const float atx = out[TXX * P + co], atz = out[TZZ * P + co], atxz = out[TXZ * P + co];
        float dzp_vx, dxm_vz, dxp_vx, dzm_vz, dzp_tz, dxm_tx, dxp_txz, dzm_txz;
        float vx = 0.f, vz = 0.f, tx = 0.f, tz = 0.f, txz = 0.f;
        if constexpr (!QD) {
        if (F) {
            // DzpVx is formed from vz, as the reference does (elastic.cl:485)
            dzp_vx = wfwd<R>(wvz, a.k.cz);
            dxm_vz = gbwd<R>(F + VZ * P, co, 1, a.k.cx);
            dxp_vx = gfwd<R>(F + VX * P, co, 1, a.k.cx);
            dzm_vz = wbwd<R>(wvz, a.k.cz);
            dzp_tz = wfwd<R>(wtz, a.k.cz);
            dxm_tx = gbwd<R>(F + TXX * P, co, 1, a.k.cx);
            dxp_txz = gfwd<R>(F + TXZ * P, co, 1, a.k.cx);
            dzm_txz = wbwd<R>(wtxz, a.k.cz);
            if (ENERGY) {
                vx = F[VX * P + co];
                vz = wvz[R];
                tx = F[TXX * P + co];
                tz = wtz[R];
                txz = wtxz[R];
            }
        } else {
#define B16F(f, k) bf(F16 + (f) * P, (k))
#define BFWD(f, s)                                                                                       \
    (a.k.c##s[0] * (B16F(f, co + st) - B16F(f, co)) + a.k.c##s[1] * (B16F(f, co + 2 * st) - B16F(f, co - st)) + \
     (R == 4 ? a.k.c##s[2] * (B16F(f, co + 3 * st) - B16F(f, co - 2 * st)) +                              \
                   a.k.c##s[3] * (B16F(f, co + 4 * st) - B16F(f, co - 3 * st))                            \
             : 0.f))
#define BBWD(f, s)                                                                                       \
    (a.k.c##s[0] * (B16F(f, co) - B16F(f, co - st)) + a.k.c##s[1] * (B16F(f, co + st) - B16F(f, co - 2 * st)) + \
     (R == 4 ? a.k.c##s[2] * (B16F(f, co + 2 * st) - B16F(f, co - 3 * st)) +                              \
                   a.k.c##s[3] * (B16F(f, co + 3 * st) - B16F(f, co - 4 * st))                            \
             : 0.f))
            long long st = sz_;
            dzp_vx = BFWD(VZ, z);
            dzm_vz = BBWD(VZ, z);
            dzp_tz = BFWD(TZZ, z);
            dzm_txz = BBWD(TXZ, z);
            st = 1;
            dxm_vz = BBWD(VZ, x);
            dxp_vx = BFWD(VX, x);
            dxm_tx = BBWD(TXX, x);
            dxp_txz = BFWD(TXZ, x);
            if (ENERGY) {
                vx = B16F(VX, co);
                vz = B16F(VZ, co);
                tx = B16F(TXX, co);
                tz = B16F(TZZ, co);
                txz = B16F(TXZ, co);
            }
#undef B16F
#undef BFWD
#undef BBWD
        }
        }
        const float b = __ldg(a.mat + 2 * P + co);
        if constexpr (QD) {
            const unsigned char *F8 = QD == 2 ? a.fwd8 + slot * a.fwd_stride : nullptr;
            const float q0 = qld<QD>(F, F16, F8, Q_DXP_VX * P + co), q1 = qld<QD>(F, F16, F8, Q_DZM_VZ * P + co),
                        q2 = qld<QD>(F, F16, F8, Q_VZS * P + co), q3 = qld<QD>(F, F16, F8, Q_TXS * P + co),
                        q4 = qld<QD>(F, F16, F8, Q_TZS * P + co);
            float gmu = G[0 * P + co], glam = G[1 * P + co], grho = G[2 * P + co];
            gmu += 2.f * dt * (atx * q0 + atz * q1) + dt * atxz * q2;
            glam += dt * (atx + atz) * (q0 + q1);
            grho += -(dt * (b * b)) * (avx * q3 + avz * q4);
            G[0 * P + co] = gmu;
            G[1 * P + co] = glam;
            G[2 * P + co] = grho;
        } else {
        float gmu = PF ? s_g[(0 * TZ + r) * TX + c] : G[0 * P + co];
        float glam = PF ? s_g[(1 * TZ + r) * TX + c] : G[1 * P + co];
        float grho = PF ? s_g[(2 * TZ + r) * TX + c] : G[2 * P + co];
        gmu += 2.f * dt * (atx * dxp_vx + atz * dzm_vz) + dt * atxz * (dzp_vx + dxm_vz);
        glam += dt * (atx + atz) * (dxp_vx + dzm_vz);
        grho += -(dt * (b * b)) * (avx * (dxm_tx + dzm_txz) + avz * (dzp_tz + dxp_txz));
        G[0 * P + co] = gmu;
        G[1 * P + co] = glam;
        G[2 * P + co] = grho;
        if (ENERGY) {
            float dt2 = dt * dt;
            G[3 * P + co] += 4.f * dt2 * (tx * tx * dxp_vx * dxp_vx + tz * tz * dzm_vz * dzm_vz) +
                             dt2 * txz * txz * (dzp_vx * dzp_vx + dxm_vz * dxm_vz);
            G[4 * P + co] += dt2 * (tx * tx + tz * tz) * (dxp_vx * dxp_vx + dzm_vz * dzm_vz);
            G[5 * P + co] += dt2 * (vx * vx * (dxm_tx * dxm_tx + dzm_txz * dzm_txz) +
                                    vz * vz * (dzp_tz * dzp_tz + dxp_txz * dxp_txz));
        }
        }
        }
        // the residual the next step injects (Adj_injSrc, elastic_surface.cl:48-71),
        // added to this step's output after the imaging has read it
        if (a.epi_row >= 0) inject_epilogue(a, a.epi_row, slot, gi, gj, co, avx, avz, out);
        out[VX * P + co] = avx;
        out[VZ * P + co] = avz;
    }
}

// The stress planes (Q_TXS, Q_TZS) of the difference set of state S: for
// the last state of a forward run or a recomputed segment, which no later
// forward step reads.  The imaging domain of every slot; one thread per
// cell, grid (ceil(tnx / 256), tnz, slots).
template <int R, int QD>
__global__ void __launch_bounds__(256) qstress_kernel(Grid g, Coef k, const float *in, long long in_stride, void *q,
                                                      unsigned char *q8, long long q_stride, int npml)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    const int glo = npml + R;
    if (i < glo || i > g.tnz - R - npml || j < glo || j > g.tnx - R - npml) return;
    const long long P = g.plane, co = cell_off(g, i, j), qo = blockIdx.z * q_stride + co;
    const float *S = in + blockIdx.z * in_stride;
    qst1<QD>(q, q8, qo + Q_TXS * P, gbwd<R>(S + TXX * P, co, 1, k.cx) + gbwd<R>(S + TXZ * P, co, g.pitch, k.cz));
    qst1<QD>(q, q8, qo + Q_TZS * P, gfwd<R>(S + TZZ * P, co, g.pitch, k.cz) + gfwd<R>(S + TXZ * P, co, 1, k.cx));
}

// ---------------------------------------------------------------------------
// exact discrete adjoint (no counterpart in the reference): the transpose of
// fwd_step, so the accumulated gradient is the exact derivative of
// J = 1/2 sum (traces - observed)^2 with respect to lam, mu and the buoyancy
// b, the damping profiles held fixed.  Uses (D+)^T = -D- and (D-)^T = -D+ on
// fields that vanish outside the update domain.  Per step t, from the adjoint
// L_{t+1} of S_{t+1}:
//   a  = (1 - dt d) L_tau                          (stress update, in D)
//   P1 = dt((lam+2mu) a_xx + lam a_zz), P2 = dt mu a_xz, P3 = dt(lam a_xx + (lam+2mu) a_zz)
//   m_vx = L_vx - Dx-(P1) - Dz-(P2),  m_vz = L_vz - Dz+(P3) - Dx+(P2)
//   B  = (1 - dt d) m_v                            (velocity update, in D)
//   Q1 = dt b B_vx, Q2 = dt b B_vz
//   L_t: v = B (in D, else m), txx = a - Dx+(Q1), tzz = a - Dz-(Q2), txz = a - Dz+(Q1) - Dx-(Q2)
//   Glam += dt (a_xx + a_zz)(Dx+ vx + Dz- vz)            [velocities of S_{t+1}]
//   Gmu  += dt (2 a_xx Dx+ vx + 2 a_zz Dz- vz + a_xz (Dx- vz + Dz+ vx))
//   Gb   += dt (B_vx (Dx- txx + Dz- txz) + B_vz (Dz+ tzz + Dx+ txz))  [stresses of S_t + source]
// The trace adjoint (dJ/dtrace into L_t at the receivers) is a separate
// inject_kernel launch after the step.
// ---------------------------------------------------------------------------
struct ExactArgs {
    Grid g;
    Coef k;
    const float *in;        // L_{t+1}, slot 0
    float *out;             // L_t
    long long in_stride, out_stride;
    const float *s1, *s0;   // forward states S_{t+1}, S_t, slot 0 (FP32)
    long long s1_stride, s0_stride;
    // BF16 or 24-bit snapshots instead (kernel instance BF): S_{t+1} always,
    // S_t when s0h is set (else S_t is the FP32 restart state s0, rounded to
    // the snapshot format as it is read); s1b / s0b: the byte planes of
    // 24-bit snapshots (NULL for BF16)
    const __nv_bfloat16 *s1h, *s0h;
    const unsigned char *s1b, *s0b;
    const float *mat;       // lam, mu, b, rho planes
    const float *dampx, *dampz;
    float *gacc;            // [slot][3][plane]: Glam, Gmu, Gb
    long long gacc_stride;
    int shot0;
    const int *srcx, *srcz;
    float4 src;             // source sample added to S_t at this step
    int add_src;
};

// Coefficient of f[j + o] in a backward / forward difference at j.
template <int R>
__device__ __forceinline__ float coef_bwd(int o, const float *c)
{
    return (o >= 0 && o < R) ? c[o] : ((o < 0 && o >= -R) ? -c[-o - 1] : 0.f);
}

template <int R>
__device__ __forceinline__ float coef_fwd(int o, const float *c)
{
    return (o >= 1 && o <= R) ? c[o - 1] : ((o <= 0 && o > -R) ? -c[-o] : 0.f);
}

template <int R, int TZ>
struct ExactShape {
    static constexpr int PW = TX + 4 * R, PH = TZ + 4 * R;  // P fields: tile +- 2R
    static constexpr int QW = TX + 2 * R, QH = TZ + 2 * R;  // Q fields: tile +- R
    static constexpr int FLOATS = 3 * PW * PH + 2 * QW * QH;
};

template <int R, int TZ, bool BF>
__global__ void __launch_bounds__(NTHREADS) exact_adj_step(const __grid_constant__ ExactArgs a)
{
    using S = ExactShape<R, TZ>;
    constexpr int PW = S::PW, PH = S::PH, QW = S::QW, QH = S::QH;
    extern __shared__ float4 smem4[];
    float *p1 = reinterpret_cast<float *>(smem4), *p2 = p1 + PH * PW, *p3 = p2 + PH * PW;
    float *q1 = p3 + PH * PW, *q2 = q1 + QH * QW;

    const Grid &g = a.g;
    const long long P = g.plane;
    const int slot = blockIdx.z, shot = a.shot0 + slot;
    const int j0 = blockIdx.x * TX, i0 = blockIdx.y * TZ;
    const float *L1 = a.in + slot * a.in_stride;
    float *L0 = a.out + slot * a.out_stride;
    const float *S1 = BF ? nullptr : a.s1 + slot * a.s1_stride;
    const float *S0 = (BF && a.s0h) ? nullptr : a.s0 + slot * a.s0_stride;
    const __nv_bfloat16 *H1 = BF ? a.s1h + slot * a.s1_stride : nullptr;
    const __nv_bfloat16 *H0 = (BF && a.s0h) ? a.s0h + slot * a.s0_stride : nullptr;
    const unsigned char *B1 = (BF && a.s1b) ? a.s1b + slot * a.s1_stride : nullptr;
    const unsigned char *B0 = (BF && a.s0b) ? a.s0b + slot * a.s0_stride : nullptr;
    const bool x24 = a.s1b != nullptr;  // 24-bit snapshots
    float *G = a.gacc + slot * a.gacc_stride;
    const float dt = a.k.dt;

    // stress update, transposed
    for (int e = threadIdx.x; e < PH * PW; e += NTHREADS) {
        const int r = e / PW, c = e - r * PW, i = i0 - 2 * R + r, j = j0 - 2 * R + c;
        float v1 = 0.f, v2 = 0.f, v3 = 0.f;
        if (in_domain(g, R, i, j)) {
            const long long co = cell_off(g, i, j);
            const float damp = 1.f - dt * (__ldg(a.dampx + j + XO) + __ldg(a.dampz + i + ZO));
            const float axx = damp * __ldg(L1 + TXX * P + co), azz = damp * __ldg(L1 + TZZ * P + co),
                        axz = damp * __ldg(L1 + TXZ * P + co);
            const float lam = __ldg(a.mat + co), mu = __ldg(a.mat + P + co), l2m = lam + 2.f * mu;
            v1 = dt * (l2m * axx + lam * azz);
            v2 = dt * (mu * axz);
            v3 = dt * (lam * axx + l2m * azz);
        }
        p1[e] = v1;
        p2[e] = v2;
        p3[e] = v3;
    }
    __syncthreads();

    // velocity update, transposed
    for (int e = threadIdx.x; e < QH * QW; e += NTHREADS) {
        const int r = e / QW, c = e - r * QW, i = i0 - R + r, j = j0 - R + c;
        float v1 = 0.f, v2 = 0.f;
        if (in_domain(g, R, i, j)) {
            const long long co = cell_off(g, i, j);
            const int ip = (r + R) * PW + c + R;
            const float mvx = __ldg(L1 + VX * P + co) - dbwd<R>(p1, ip, 1, a.k.cx) - dbwd<R>(p2, ip, PW, a.k.cz);
            const float mvz = __ldg(L1 + VZ * P + co) - dfwd<R>(p3, ip, PW, a.k.cz) - dfwd<R>(p2, ip, 1, a.k.cx);
            const float damp = 1.f - dt * (__ldg(a.dampx + j + XO) + __ldg(a.dampz + i + ZO));
            const float b = __ldg(a.mat + 2 * P + co);
            v1 = dt * (b * (damp * mvx));
            v2 = dt * (b * (damp * mvz));
        }
        q1[e] = v1;
        q2[e] = v2;
    }
    __syncthreads();

    // the tile: L_t and the gradients
    const int si = a.add_src ? a.srcz[shot] : -(1 << 30), sj = a.srcx[shot];
    for (int e = threadIdx.x; e < TZ * TX; e += NTHREADS) {
        const int r = e / TX, c = e - r * TX, i = i0 + r, j = j0 + c;
        if (i >= g.tnz || j >= g.tnx) continue;
        const long long co = cell_off(g, i, j);
        const int ip = (r + 2 * R) * PW + c + 2 * R, iq = (r + R) * QW + c + R;
        const bool dom = in_domain(g, R, i, j);
        const float damp = dom ? 1.f - dt * (__ldg(a.dampx + j + XO) + __ldg(a.dampz + i + ZO)) : 1.f;
        const float mvx = __ldg(L1 + VX * P + co) - dbwd<R>(p1, ip, 1, a.k.cx) - dbwd<R>(p2, ip, PW, a.k.cz);
        const float mvz = __ldg(L1 + VZ * P + co) - dfwd<R>(p3, ip, PW, a.k.cz) - dfwd<R>(p2, ip, 1, a.k.cx);
        const float bvx = damp * mvx, bvz = damp * mvz;
        const float axx = damp * __ldg(L1 + TXX * P + co), azz = damp * __ldg(L1 + TZZ * P + co),
                    axz = damp * __ldg(L1 + TXZ * P + co);
        L0[VX * P + co] = bvx;
        L0[VZ * P + co] = bvz;
        L0[TXX * P + co] = axx - dfwd<R>(q1, iq, 1, a.k.cx);
        L0[TZZ * P + co] = azz - dbwd<R>(q2, iq, QW, a.k.cz);
        L0[TXZ * P + co] = axz - dfwd<R>(q1, iq, QW, a.k.cz) - dbwd<R>(q2, iq, 1, a.k.cx);
        if (!dom) continue;
        const long long pz = g.pitch;
        // velocity differences of S_{t+1}, stress differences of S_t; ld(f)
        // gives the loader of field f's plane
        auto vdiffs = [&](auto ld, float &xp_vx, float &zm_vz, float &xm_vz, float &zp_vx) {
            xp_vx = lfwd<R>(ld(VX), co, 1, a.k.cx);
            zm_vz = lbwd<R>(ld(VZ), co, pz, a.k.cz);
            xm_vz = lbwd<R>(ld(VZ), co, 1, a.k.cx);
            zp_vx = lfwd<R>(ld(VX), co, pz, a.k.cz);
        };
        auto sdiffs = [&](auto ld, float &xm_tx, float &zm_txz, float &zp_tz, float &xp_txz) {
            xm_tx = lbwd<R>(ld(TXX), co, 1, a.k.cx);
            zm_txz = lbwd<R>(ld(TXZ), co, pz, a.k.cz);
            zp_tz = lfwd<R>(ld(TZZ), co, pz, a.k.cz);
            xp_txz = lfwd<R>(ld(TXZ), co, 1, a.k.cx);
        };
        auto f32 = [&](const float *S) {
            return [=](int f) { return [=](long long i) { return __ldg(S + f * P + i); }; };
        };
        auto snap = [&](const __nv_bfloat16 *S, const unsigned char *B) {
            return [=](int f) { return [=](long long i) { return snapv(S, B, f * P + i); }; };
        };
        auto f32_as_snap = [&](const float *S) {
            return [=](int f) {
                return [=](long long i) {
                    const float v = __ldg(S + f * P + i);
                    return x24 ? fp24_round(v) : __bfloat162float(__float2bfloat16_rn(v));
                };
            };
        };
        float dxp_vx, dzm_vz, dxm_vz, dzp_vx, dxm_tx, dzm_txz, dzp_tz, dxp_txz;
        if (BF) {
            vdiffs(snap(H1, B1), dxp_vx, dzm_vz, dxm_vz, dzp_vx);
            if (H0)
                sdiffs(snap(H0, B0), dxm_tx, dzm_txz, dzp_tz, dxp_txz);
            else
                sdiffs(f32_as_snap(S0), dxm_tx, dzm_txz, dzp_tz, dxp_txz);
        } else {
            vdiffs(f32(S1), dxp_vx, dzm_vz, dxm_vz, dzp_vx);
            sdiffs(f32(S0), dxm_tx, dzm_txz, dzp_tz, dxp_txz);
        }
        if (si == i) dxm_tx = fmaf(coef_bwd<R>(sj - j, a.k.cx), a.src.z, dxm_tx);  // S_t + source
        if (sj == j) dzp_tz = fmaf(coef_fwd<R>(si - i, a.k.cz), a.src.w, dzp_tz);
        G[0 * P + co] += dt * (axx + azz) * (dxp_vx + dzm_vz);
        G[1 * P + co] += dt * (2.f * axx * dxp_vx + 2.f * azz * dzm_vz + axz * (dxm_vz + dzp_vx));
        G[2 * P + co] += dt * (bvx * (dxm_tx + dzm_txz) + bvz * (dzp_tz + dxp_txz));
    }
}

// Exact gradient on the model grid: the three padded accumulators summed
// over the cells each model cell was copied to (edge-replicated padding,
// fwi_tools.py:776-811), then the chain rule lam = rho vp^2 - 2 mu,
// mu = rho vs^2, b = 1/rho.  param 0: (lam, mu, rho) with rho at fixed
// lam, mu; 1: (vp, vs, rho).
__global__ void exact_post_kernel(Grid g, int nz, int nx, int npml, const float *gacc, const float *mat, int param,
                                  float *out)
{
    const long long n = (long long)nz * nx, P = g.plane;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e / nx), j = (int)(e - (long long)i * nx);
        const int r0 = i == 0 ? 0 : i + npml, r1 = i == nz - 1 ? g.tnz - 1 : i + npml;
        const int c0 = j == 0 ? 0 : j + npml, c1 = j == nx - 1 ? g.tnx - 1 : j + npml;
        double sl = 0.0, sm = 0.0, sb = 0.0;
        for (int r = r0; r <= r1; ++r)
            for (int c = c0; c <= c1; ++c) {
                const long long co = cell_off(g, r, c);
                sl += gacc[co];
                sm += gacc[P + co];
                sb += gacc[2 * P + co];
            }
        const long long cm = cell_off(g, i + npml, j + npml);
        const double lam = mat[cm], mu = mat[P + cm], rho = mat[3 * P + cm];
        const double grho_lm = -sb / (rho * rho);  // d/drho at fixed lam, mu: b = 1/rho
        if (param == 0) {
            out[e] = (float)sl;
            out[n + e] = (float)sm;
            out[2 * n + e] = (float)grho_lm;
        } else {
            const double vp = sqrt((lam + 2.0 * mu) / rho), vs = sqrt(mu / rho);
            out[e] = (float)(2.0 * rho * vp * sl);
            out[n + e] = (float)(-4.0 * rho * vs * sl + 2.0 * rho * vs * sm);
            out[2 * n + e] = (float)((vp * vp - 2.0 * vs * vs) * sl + vs * vs * sm + grho_lm);
        }
    }
}

// ---------------------------------------------------------------------------
// set-up and post-processing kernels
// ---------------------------------------------------------------------------

// max(vp) as the bits of a non-negative float (atomicMax on int orders them).
__global__ void vp_max_kernel(const float *vp, long long n, int *out_bits)
{
    float m = 0.f;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, vp[k]);
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_int(m));
}

// Materials of the padded grid (fwi_tools.py:776-811 padding,
// wave_propagation.py:575-591).  float32 with explicit rounding so the
// values match numpy's elementwise float32 results bit for bit.
__global__ void model_kernel(Grid g, int nz, int nx, int npml, const float *vp, const float *vs, const float *rho,
                             float *mat)
{
    long long n = (long long)g.tnz * g.tnx;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        int i = (int)(k / g.tnx), j = (int)(k - (long long)i * g.tnx);
        int mi = min(max(i - npml, 0), nz - 1), mj = min(max(j - npml, 0), nx - 1);
        long long m = (long long)mi * nx + mj;
        float p = vp[m], s = vs[m], r = rho[m];
        float mu = __fmul_rn(r, __fmul_rn(s, s));
        float lam = __fsub_rn(__fmul_rn(r, __fmul_rn(p, p)), __fmul_rn(2.f, mu));
        long long c = cell_off(g, i, j);
        mat[c] = lam;
        mat[g.plane + c] = mu;
        mat[2 * g.plane + c] = __frcp_rn(r);
        mat[3 * g.plane + c] = r;
    }
}

__global__ void damp_kernel(Grid g, const float *damp_x, const float *damp_z, const int *vpmax_bits, float *dampx,
                            float *dampz)
{
    float vmax = __int_as_float(*vpmax_bits);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.pitch + g.rows; k += gridDim.x * blockDim.x) {
        if (k < g.pitch) {
            int j = k - XO;
            dampx[k] = (j >= 0 && j < g.tnx) ? __fmul_rn(damp_x[j], vmax) : 0.f;
        } else {
            int i = k - g.pitch - ZO;
            dampz[k - g.pitch] = (i >= 0 && i < g.tnz) ? __fmul_rn(damp_z[i], vmax) : 0.f;
        }
    }
}

// Sum the per-slot accumulators into slot 0: G0 += G1 + ... (shot order).
__global__ void reduce_slots_kernel(float *gacc, long long slot_stride, int nslots, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        float s = gacc[k];
        for (int q = 1; q < nslots; ++q) s += gacc[q * slot_stride + k];
        gacc[k] = s;
    }
}

// Copy the padded accumulators out as dense [nacc][tnz][tnx].
__global__ void raw_out_kernel(Grid g, const float *gacc, int nacc, float *raw)
{
    long long n = (long long)g.tnz * g.tnx;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n * nacc;
         k += (long long)gridDim.x * blockDim.x) {
        int q = (int)(k / n);
        long long r = k - q * n;
        int i = (int)(r / g.tnx), j = (int)(r - (long long)i * g.tnx);
        raw[k] = gacc[q * g.plane + cell_off(g, i, j)];
    }
}

// Energy-balancing factor 1/sqrt(P) inside the window, its max |.| as bits.
struct PostArgs {
    Grid g;
    int nz, nx, npml;
    int r0, r1, c0, c1;  // window (model grid)
    int energy;
    int param;           // 0 lmd, 1 dv
    const float *gacc;   // slot 0 accumulators
    const float *mat;
    int *fmax_bits;      // [3] max factor per gradient (Gmu, Glam, Grho order)
    float *out;          // [3][nz][nx]
};

__device__ __forceinline__ float window_factor(const PostArgs &a, int q, int i, int j)
{
    // q: 0 Gmu, 1 Glam, 2 Grho ; returns 1/sqrt(P) (or 1) inside, 0 outside
    if (i < a.r0 || i >= a.r1 || j < a.c0 || j >= a.c1) return 0.f;
    if (!a.energy) return 1.f;
    float p = a.gacc[(3 + q) * a.g.plane + cell_off(a.g, i + a.npml, j + a.npml)];
    return __fdiv_rn(1.f, __fsqrt_rn(p));
}

__global__ void factor_max_kernel(PostArgs a)
{
    float m[3] = {0.f, 0.f, 0.f};
    long long n = (long long)a.nz * a.nx;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        int i = (int)(k / a.nx), j = (int)(k - (long long)i * a.nx);
        for (int q = 0; q < 3; ++q) m[q] = fmaxf(m[q], fabsf(window_factor(a, q, i, j)));
    }
    for (int q = 0; q < 3; ++q) {
        float v = m[q];
        for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0) atomicMax(a.fmax_bits + q, __float_as_int(v));
    }
}

// gradient_reading + grad_lmd_to_vd (wave_propagation.py:279-331,
// grad_switcher.py:331-383) with numpy's float32 operation order.
__global__ void post_kernel(PostArgs a)
{
    long long n = (long long)a.nz * a.nx;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        int i = (int)(k / a.nx), j = (int)(k - (long long)i * a.nx);
        long long c = cell_off(a.g, i + a.npml, j + a.npml);
        float gm = a.gacc[0 * a.g.plane + c], gl = a.gacc[1 * a.g.plane + c], gr = a.gacc[2 * a.g.plane + c];
        float fmu = __fdiv_rn(window_factor(a, 0, i, j), __int_as_float(a.fmax_bits[0]));
        float flam = __fdiv_rn(window_factor(a, 1, i, j), __int_as_float(a.fmax_bits[1]));
        float frho = __fdiv_rn(window_factor(a, 2, i, j), __int_as_float(a.fmax_bits[2]));
        float glam = __fmul_rn(gl, flam), gmu = __fmul_rn(gm, fmu), grho = __fmul_rn(gr, frho);
        if (a.param == 0) {
            a.out[k] = glam;
            a.out[n + k] = gmu;
            a.out[2 * n + k] = grho;
            continue;
        }
        float lam = a.mat[c], mu = a.mat[a.g.plane + c], rho = a.mat[3 * a.g.plane + c];
        float vp = __fsqrt_rn(__fdiv_rn(__fadd_rn(lam, __fmul_rn(2.f, mu)), rho));
        float vs = __fsqrt_rn(__fdiv_rn(mu, rho));
        float vs2 = __fmul_rn(vs, vs);
        float vpvs = __fsub_rn(__fmul_rn(vp, vp), __fmul_rn(2.f, __fmul_rn(vs, vs)));
        float gvp = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(__fmul_rn(glam, 2.f), vp), rho), __fmul_rn(gmu, 0.f)),
                              __fmul_rn(grho, 0.f));
        float gvs = __fadd_rn(__fadd_rn(__fmul_rn(glam, __fmul_rn(__fmul_rn(-4.f, rho), vs)),
                                        __fmul_rn(__fmul_rn(__fmul_rn(gmu, 2.f), vs), rho)),
                              __fmul_rn(grho, 0.f));
        float grr = __fadd_rn(__fadd_rn(__fmul_rn(glam, vpvs), __fmul_rn(gmu, vs2)), grho);
        a.out[k] = gvp;
        a.out[n + k] = gvs;
        a.out[2 * n + k] = grr;
    }
}

// Sums that do not depend on scheduling: each block writes its partial sum
// (a fixed tree over its threads) to partials[blockIdx.x]; one warp then adds
// the partials in a fixed order.  Equal inputs give equal bits, so a line
// search comparing two evaluations of the same model sees a tie as a tie.
__device__ __forceinline__ void block_partial(double acc, double *partials)
{
    __shared__ double warp_sums[32];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += warp_sums[w];
        partials[blockIdx.x] = t;
    }
}

// total += 0.5 * sum(partials[0..n)), one warp
__global__ void sum_partials_kernel(const double *partials, int n, double *total)
{
    double acc = 0.0;
    for (int k = threadIdx.x; k < n; k += 32) acc += partials[k];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) *total += 0.5 * acc;
}

// res = est - obs; partials[block] = this block's share of sum(res^2)
__global__ void l2_kernel(const float *est, const float *obs, float *res, long long n, double *partials)
{
    double acc = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        float r = __fsub_rn(est[k], obs[k]);
        res[k] = r;
        acc += (double)r * (double)r;
    }
    block_partial(acc, partials);
}

// L2 misfit of one shot group's columns of the traces (CostFunction.l2,
// fwi_tools.py:1402-1422, on the section of acquisition.py:313-333) and the
// adjoint sources of those columns.  mean_stress: the two stress keys both
// hold (txx + tzz) / 2; their residuals are the reference's adjoint sources
// for txx and tzz (prepare_residual, processing.py:142-158), and for the
// exact adjoint each stress field gets half their sum (the derivative of the
// misfit through the mean).
struct MisfitArgs {
    const float *traces;   // [5][nt][ncol]
    const float *obs[5];   // nullable per field: not in the misfit
    float *res[5];
    long long nt, ncol, col0, ncols, plane;
    int mean_stress, exact;
    double *partials;      // one per block (block_partial)
};

__global__ void misfit_kernel(const MisfitArgs m)
{
    double acc = 0.0;
    const long long n = m.nt * m.ncols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long t = e / m.ncols, o = t * m.ncol + m.col0 + (e - t * m.ncols);
        if (m.mean_stress) {
            const float mean = __fdiv_rn(__fadd_rn(m.traces[TXX * m.plane + o], m.traces[TZZ * m.plane + o]), 2.f);
            const float r1 = m.obs[TXX] ? __fsub_rn(mean, m.obs[TXX][o]) : 0.f;
            const float r2 = m.obs[TZZ] ? __fsub_rn(mean, m.obs[TZZ][o]) : 0.f;
            acc += (double)r1 * r1 + (double)r2 * r2;
            if (m.exact) {
                const float h = 0.5f * (r1 + r2);
                m.res[TXX][o] = h;
                m.res[TZZ][o] = h;
            } else {
                if (m.obs[TXX]) m.res[TXX][o] = r1;
                if (m.obs[TZZ]) m.res[TZZ][o] = r2;
            }
        }
        for (int f = 0; f < 5; ++f) {
            if (!m.obs[f] || (m.mean_stress && (f == TXX || f == TZZ))) continue;
            const float r = __fsub_rn(m.traces[f * m.plane + o], m.obs[f][o]);
            m.res[f][o] = r;
            acc += (double)r * r;
        }
    }
    block_partial(acc, m.partials);
}

__global__ void mean2_kernel(const float *a, const float *b, float *out, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        out[k] = __fdiv_rn(__fadd_rn(a[k], b[k]), 2.f);
}

// Gaussian smoothing of the gradient (gaussian_filter, wave_propagation.py:
// 923-936): a 1-D correlation with normalised Gaussian weights along one axis
// of `n` stacked (nz, nx) arrays, edges extended by half-sample reflection
// (d c b a | a b c d | d c b a), sums in double, result rounded to float.
constexpr int SMOOTH_MAX_RADIUS = 127;
struct SmoothWeights {
    double w[2 * SMOOTH_MAX_RADIUS + 1];
};

__device__ __forceinline__ int reflect_index(int i, int n)
{
    const int p = 2 * n;
    int m = i % p;
    if (m < 0) m += p;
    return m < n ? m : p - 1 - m;
}

__global__ void smooth_kernel(const float *in, float *out, int n, int nz, int nx, int axis, int radius,
                              const __grid_constant__ SmoothWeights W)
{
    const long long total = (long long)n * nz * nx;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long plane = e / ((long long)nz * nx);
        const int rem = (int)(e - plane * nz * nx), i = rem / nx, j = rem - i * nx;
        const float *src = in + plane * nz * nx;
        double acc = 0.0;
        for (int k = -radius; k <= radius; ++k) {
            const float v = axis == 0 ? src[(long long)reflect_index(i + k, nz) * nx + j]
                                      : src[(long long)i * nx + reflect_index(j + k, nx)];
            acc += W.w[k + radius] * (double)v;
        }
        out[e] = (float)acc;
    }
}

}  // namespace pyfwi
