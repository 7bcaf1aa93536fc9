/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle.
 *
 * A plain-C restatement of PyFWI's 2-D isotropic-elastic velocity-stress
 * staggered-grid propagator and of its adjoint-state gradient, used as the
 * checker for the CUDA product path.  Only tests/, __graft_entry__.smoke() and
 * the cpu_baseline leg of bench.py may load it; the product never does.
 *
 * Semantics follow the reference kernels (PyFWI, src/PyFWI/elastic.cl,
 * elastic_surface.cl, elastic_crosswell.cl) and the host loops of
 * src/PyFWI/wave_propagation.py:
 *   - fields are flat row-major arrays, idx = i*Nx + j (wave_propagation.py:452);
 *     x-neighbours wrap into the adjacent row exactly as the flat index does,
 *     and reads past either end of an array land in a zero guard band that the
 *     caller allocates (>= 4*Nx+4 elements before and after every field);
 *   - the scalars dt, dx, dz, c1..c4 are the reference's "%f" macro values and
 *     are kept as double, so with REAL=float the arithmetic promotes to double
 *     and rounds on store, as an OpenCL C compiler with fp64 does with the
 *     reference's unsuffixed literals (wave_propagation.py:434-490);
 *   - build with REAL=double for the FP64 oracle.
 * Build: oracle/Makefile (gcc -O3 -fopenmp -ffp-contract=off).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL float
#endif

typedef struct {
    int32_t Nz, Nx;          /* padded grid (tnz, tnx) */
    int32_t sdo;             /* half stencil order: 2 (4th order) or 4 (8th) */
    int32_t npml;
    double dt, dx, dz;       /* internal dt and dh after "%f" rounding */
    double c1, c2, c3, c4;   /* stencil coefficients after "%f" rounding */
    int32_t nt, dt_scale, nt_ext;
    int32_t acq_type;        /* 0 crosswell, 1 surface, 2 surface + 2 wells */
    int32_t Nr, n_main_rec, n_extera_rec, dxr;
    int32_t rec_top_left_const, rec_top_left_var;
    int32_t rec_top_right_const, rec_top_right_var;
    int32_t rec_surface_const, rec_surface_var;
} orc_cfg;

/* The eight material/field arrays a step touches.  Each pointer addresses
 * element 0 of an Nz*Nx array that has a zero guard on both sides. */
typedef struct {
    REAL *vx, *vz, *taux, *tauz, *tauxz;
} orc_state;

typedef struct {
    const REAL *lam, *mu, *rho_b;     /* rho_b = 1/rho (buoyancy) */
    const REAL *dxpml, *dzpml;        /* damping profile * vp_max, Nz*Nx */
} orc_model;

/* ---- one-sided staggered differences ------------------------------------
 * fwd: (c1(f[+1]-f[0]) + c2(f[+2]-f[-1]) + c3(f[+3]-f[-2]) + c4(f[+4]-f[-3]))/h
 * bwd: (c1(f[0]-f[-1]) + c2(f[+1]-f[-2]) + c3(f[+2]-f[-3]) + c4(f[+3]-f[-4]))/h
 * s is the flat stride of the direction (1 for x, Nx for z).  The operand
 * order and the double-valued coefficients reproduce the reference
 * expressions (elastic.cl:168-172, 208-213, 248-252, 291-295). */
static inline REAL dfwd(const REAL *f, long c, long s, const orc_cfg *g, double h)
{
    return (REAL)((g->c1 * (f[c + s] - f[c]) + g->c2 * (f[c + 2 * s] - f[c - s]) +
                   g->c3 * (f[c + 3 * s] - f[c - 2 * s]) + g->c4 * (f[c + 4 * s] - f[c - 3 * s])) / h);
}

static inline REAL dbwd(const REAL *f, long c, long s, const orc_cfg *g, double h)
{
    return (REAL)((g->c1 * (f[c] - f[c - s]) + g->c2 * (f[c + s] - f[c - 2 * s]) +
                   g->c3 * (f[c + 2 * s] - f[c - 3 * s]) + g->c4 * (f[c + 3 * s] - f[c - 4 * s])) / h);
}

/* Same differences applied to the pointwise product a*b (adjoint kernels,
 * elastic.cl:385-406). */
#define PR(a, b, k) ((a)[k] * (b)[k])
static inline REAL dfwd_p(const REAL *a, const REAL *b, long c, long s, const orc_cfg *g, double h)
{
    return (REAL)((g->c1 * (PR(a, b, c + s) - PR(a, b, c)) + g->c2 * (PR(a, b, c + 2 * s) - PR(a, b, c - s)) +
                   g->c3 * (PR(a, b, c + 3 * s) - PR(a, b, c - 2 * s)) +
                   g->c4 * (PR(a, b, c + 4 * s) - PR(a, b, c - 3 * s))) / h);
}

static inline REAL dbwd_p(const REAL *a, const REAL *b, long c, long s, const orc_cfg *g, double h)
{
    return (REAL)((g->c1 * (PR(a, b, c) - PR(a, b, c - s)) + g->c2 * (PR(a, b, c + s) - PR(a, b, c - 2 * s)) +
                   g->c3 * (PR(a, b, c + 2 * s) - PR(a, b, c - 3 * s)) +
                   g->c4 * (PR(a, b, c + 3 * s) - PR(a, b, c - 4 * s))) / h);
}

/* Differences of (lam + 2 mu) * A (elastic.cl:432-452). */
#define L2M(k) ((lam[k] + 2 * mu[k]) * A[k])
static inline REAL dfwd_l2m(const REAL *lam, const REAL *mu, const REAL *A, long c, long s,
                            const orc_cfg *g, double h)
{
    return (REAL)((g->c1 * (L2M(c + s) - L2M(c)) + g->c2 * (L2M(c + 2 * s) - L2M(c - s)) +
                   g->c3 * (L2M(c + 3 * s) - L2M(c - 2 * s)) + g->c4 * (L2M(c + 4 * s) - L2M(c - 3 * s))) / h);
}

static inline REAL dbwd_l2m(const REAL *lam, const REAL *mu, const REAL *A, long c, long s,
                            const orc_cfg *g, double h)
{
    return (REAL)((g->c1 * (L2M(c) - L2M(c - s)) + g->c2 * (L2M(c + s) - L2M(c - 2 * s)) +
                   g->c3 * (L2M(c + 2 * s) - L2M(c - 3 * s)) + g->c4 * (L2M(c + 3 * s) - L2M(c - 4 * s))) / h);
}

/* Update domain of every propagation kernel: rows and columns sdo..N-sdo
 * inclusive (elastic.cl:163-166). */
#define FOR_DOMAIN(g)                                                   \
    _Pragma("omp parallel for schedule(static)")                        \
    for (long i = (g)->sdo; i <= (long)(g)->Nz - (g)->sdo; ++i)         \
        for (long j = (g)->sdo; j <= (long)(g)->Nx - (g)->sdo; ++j)

/* ---- forward / reverse-time propagation ---------------------------------
 * coeff=+1: update then damp (forward); coeff=-1: damp then subtract the
 * update (reverse-time reconstruction).  elastic.cl:155-308. */
void orc_update_velx(const orc_cfg *g, int coeff, orc_state *S, const orc_model *M)
{
    const long Nx = g->Nx;
    FOR_DOMAIN(g) {
        long c = i * Nx + j;
        REAL DxmTx = dbwd(S->taux, c, 1, g, g->dx);
        REAL DzmTxz = dbwd(S->tauxz, c, Nx, g, g->dz);
        if (coeff == 1) {
            S->vx[c] += coeff * g->dt * (M->rho_b[c] * (DxmTx + DzmTxz));
            S->vx[c] += coeff * g->dt * (-(M->dxpml[c] + M->dzpml[c]) * S->vx[c]);
        } else if (coeff == -1) {
            S->vx[c] += coeff * g->dt * (+(M->dxpml[c] + M->dzpml[c]) * S->vx[c]);
            S->vx[c] += coeff * g->dt * (M->rho_b[c] * (DxmTx + DzmTxz));
        }
    }
}

void orc_update_velz(const orc_cfg *g, int coeff, orc_state *S, const orc_model *M)
{
    const long Nx = g->Nx;
    FOR_DOMAIN(g) {
        long c = i * Nx + j;
        REAL DxpTxz = dfwd(S->tauxz, c, 1, g, g->dx);
        REAL DzpTz = dfwd(S->tauz, c, Nx, g, g->dz);
        if (coeff == 1) {
            S->vz[c] += coeff * g->dt * (M->rho_b[c] * (DzpTz + DxpTxz));
            S->vz[c] += coeff * g->dt * (-(M->dzpml[c] + M->dxpml[c]) * S->vz[c]);
        } else if (coeff == -1) {
            S->vz[c] += coeff * g->dt * (+(M->dzpml[c] + M->dxpml[c]) * S->vz[c]);
            S->vz[c] += coeff * g->dt * (M->rho_b[c] * (DzpTz + DxpTxz));
        }
    }
}

void orc_update_tauz(const orc_cfg *g, int coeff, orc_state *S, const orc_model *M)
{
    const long Nx = g->Nx;
    FOR_DOMAIN(g) {
        long c = i * Nx + j;
        REAL DxpVx = dfwd(S->vx, c, 1, g, g->dx);
        REAL DzmVz = dbwd(S->vz, c, Nx, g, g->dz);
        REAL lam = M->lam[c], mu = M->mu[c], d = M->dxpml[c] + M->dzpml[c];
        if (coeff == 1) {
            S->taux[c] += coeff * g->dt * ((lam + 2 * mu) * DxpVx + lam * DzmVz);
            S->tauz[c] += coeff * g->dt * ((lam + 2 * mu) * DzmVz + lam * DxpVx);
            S->taux[c] += coeff * g->dt * (-d * S->taux[c]);
            S->tauz[c] += coeff * g->dt * (-d * S->tauz[c]);
        } else if (coeff == -1) {
            S->taux[c] += coeff * g->dt * (+d * S->taux[c]);
            S->tauz[c] += coeff * g->dt * (+d * S->tauz[c]);
            S->taux[c] += coeff * g->dt * ((lam + 2 * mu) * DxpVx + lam * DzmVz);
            S->tauz[c] += coeff * g->dt * ((lam + 2 * mu) * DzmVz + lam * DxpVx);
        }
    }
}

void orc_update_tauxz(const orc_cfg *g, int coeff, orc_state *S, const orc_model *M)
{
    const long Nx = g->Nx;
    FOR_DOMAIN(g) {
        long c = i * Nx + j;
        REAL DxmVz = dbwd(S->vz, c, 1, g, g->dx);
        REAL DzpVx = dfwd(S->vx, c, Nx, g, g->dz);
        REAL d = M->dxpml[c] + M->dzpml[c];
        if (coeff == 1) {
            S->tauxz[c] += coeff * g->dt * (M->mu[c] * (DxmVz + DzpVx));
            S->tauxz[c] += coeff * g->dt * (-d * S->tauxz[c]);
        } else if (coeff == -1) {
            S->tauxz[c] += coeff * g->dt * (+d * S->tauxz[c]);
            S->tauxz[c] += coeff * g->dt * (M->mu[c] * (DxmVz + DzpVx));
        }
    }
}

/* ---- sources and receivers ----------------------------------------------
 * Record the five fields at every receiver into row `row` of seis[5][nt_ext][Nr],
 * then add the source sample at (srcz, srcx).  The reference does both in one
 * NDRange (elastic_surface.cl:7-36, elastic_crosswell.cl:1-33,
 * elastic.cl:43-98); recording before the add is the order a row-major sweep
 * of that NDRange gives whenever the receiver line starts right of column 0.
 * The crosswell variant stores vx into the vz trace, as the reference does
 * (elastic_crosswell.cl:27). */
/* Trace slots at or beyond Nr are skipped: the reference writes them into the
 * next row of its buffer, where the next recording overwrites them, or past
 * the buffer end for the last row.  A receiver cell outside the grid reads as
 * zero (the reference reads out of bounds there). */
static inline void rec5(const orc_cfg *g, const orc_state *S, REAL *seis, long row, long ir, long cell,
                        int vz_from_vx)
{
    const long plane = (long)g->nt_ext * g->Nr;
    if (ir < 0 || ir >= g->Nr) return;
    long o = row * g->Nr + ir;
    int ok = cell >= 0 && cell < (long)g->Nz * g->Nx;
    seis[0 * plane + o] = ok ? S->vx[cell] : 0;
    seis[1 * plane + o] = ok ? (vz_from_vx ? S->vx[cell] : S->vz[cell]) : 0;
    seis[2 * plane + o] = ok ? S->taux[cell] : 0;
    seis[3 * plane + o] = ok ? S->tauz[cell] : 0;
    seis[4 * plane + o] = ok ? S->tauxz[cell] : 0;
}

void orc_record(const orc_cfg *g, const orc_state *S, REAL *seis, long row)
{
    const long Nx = g->Nx, Nz = g->Nz;
    if (row < 0 || row >= g->nt_ext) return; /* reference would write past its buffer */
    if (g->acq_type == 1 || g->acq_type == 2) {
        /* surface line: work items j % dxr == 0 on row rec_surface_const */
        long i = g->rec_surface_const;
        long off = (g->acq_type == 2) ? g->n_extera_rec : 0;
        if (i >= 0 && i < Nz)
            for (long j = 0; j < Nx; j += g->dxr) {
                long ir = j / g->dxr;
                if (ir < g->n_main_rec) rec5(g, S, seis, row, off + ir, i * Nx + (j + g->rec_surface_var), 0);
            }
    }
    if (g->acq_type == 0) {
        long j = g->rec_top_right_const;
        if (j >= 0 && j < Nx)
            for (long i = 0; i < Nz; i += g->dxr) {
                long ir = i / g->dxr;
                rec5(g, S, seis, row, ir, (i + g->rec_top_right_var) * Nx + j, 1);
            }
    }
    if (g->acq_type == 2) {
        long j = g->rec_top_left_const;
        if (j >= 0 && j < Nx)
            for (long i = 0; i < Nz; i += g->dxr) {
                long ir = i / g->dxr;
                if (ir < g->n_extera_rec) rec5(g, S, seis, row, ir, (i + g->rec_top_left_var) * Nx + j, 0);
            }
        j = g->rec_top_right_const;
        long start = g->n_extera_rec + g->n_main_rec;
        if (j >= 0 && j < Nx)
            for (long i = 0; i < Nz; i += g->dxr) {
                long ir = i / g->dxr;
                rec5(g, S, seis, row, start + ir, (i + g->rec_top_right_var) * Nx + j, 0);
            }
    }
}

void orc_add_source(const orc_cfg *g, orc_state *S, long srcx, long srcz, const float *val4)
{
    if (srcz < 0 || srcz >= g->Nz || srcx < 0 || srcx >= g->Nx) return;
    long c = srcz * g->Nx + srcx;
    S->vx[c] += val4[0];
    S->vz[c] += val4[1];
    S->taux[c] += val4[2];
    S->tauz[c] += val4[3];
}

/* Add residual row (res[5][..][Nr] already sliced to this shot and row) to the
 * five adjoint fields at the receivers (elastic_surface.cl:48-71,
 * elastic_crosswell.cl:35-58, elastic.cl:316-363).  A NULL component is zero. */
/* Residual slots at or beyond Nr read as zero (the reference reads past its
 * residual buffer there), and cells outside the grid are skipped. */
static inline void inj5(const orc_cfg *g, orc_state *A, const REAL *const *res, long ir, long cell)
{
    REAL *f[5] = {A->vx, A->vz, A->taux, A->tauz, A->tauxz};
    if (ir < 0 || ir >= g->Nr || cell < 0 || cell >= (long)g->Nz * g->Nx) return;
    for (int k = 0; k < 5; ++k)
        if (res[k]) f[k][cell] += res[k][ir];
}

void orc_adj_inject(const orc_cfg *g, orc_state *A, const REAL *const *res)
{
    const long Nx = g->Nx, Nz = g->Nz;
    if (g->acq_type == 1 || g->acq_type == 2) {
        long i = g->rec_surface_const;
        long off = (g->acq_type == 2) ? g->n_extera_rec : 0;
        if (i >= 0 && i < Nz)
            for (long j = 0; j < Nx; j += g->dxr) {
                long ir = j / g->dxr;
                if (ir < g->n_main_rec) inj5(g, A, res, off + ir, i * Nx + (j + g->rec_surface_var));
            }
    }
    if (g->acq_type == 0) {
        long j = g->rec_top_right_const;
        if (j >= 0 && j < Nx)
            for (long i = 0; i < Nz; i += g->dxr) inj5(g, A, res, i / g->dxr, (i + g->rec_top_right_var) * Nx + j);
    }
    if (g->acq_type == 2) {
        long j = g->rec_top_left_const;
        if (j >= 0 && j < Nx)
            for (long i = 0; i < Nz; i += g->dxr) {
                long ir = i / g->dxr;
                if (ir < g->n_extera_rec) inj5(g, A, res, ir, (i + g->rec_top_left_var) * Nx + j);
            }
        j = g->rec_top_right_const;
        long start = g->n_extera_rec + g->n_main_rec;
        if (j >= 0 && j < Nx)
            for (long i = 0; i < Nz; i += g->dxr)
                inj5(g, A, res, start + i / g->dxr, (i + g->rec_top_right_var) * Nx + j);
    }
}

/* ---- adjoint propagation (elastic.cl:372-468) --------------------------- */
void orc_adj_update_tau(const orc_cfg *g, orc_state *A, const orc_model *M)
{
    const long Nx = g->Nx;
    FOR_DOMAIN(g) {
        long c = i * Nx + j;
        REAL DxpAVx = dfwd_p(A->vx, M->rho_b, c, 1, g, g->dx);
        REAL DzmAVz = dbwd_p(A->vz, M->rho_b, c, Nx, g, g->dz);
        A->taux[c] += -g->dt * ((M->dxpml[c]) * A->taux[c] + DxpAVx);
        A->tauz[c] += -g->dt * ((M->dzpml[c]) * A->tauz[c] + DzmAVz);
        REAL DzpAvx = dfwd_p(A->vx, M->rho_b, c, Nx, g, g->dz);
        REAL DxmAvz = dbwd_p(A->vz, M->rho_b, c, 1, g, g->dx);
        A->tauxz[c] += -g->dt * (((M->dxpml[c] + M->dzpml[c]) * A->tauxz[c]) + (DzpAvx + DxmAvz));
    }
}

void orc_adj_update_v(const orc_cfg *g, orc_state *A, const orc_model *M)
{
    const long Nx = g->Nx;
    const REAL *lam = M->lam, *mu = M->mu;
    FOR_DOMAIN(g) {
        long c = i * Nx + j;
        REAL DxmAtaux = dbwd_l2m(lam, mu, A->taux, c, 1, g, g->dx);
        REAL DxmAtauz = dbwd_p(lam, A->tauz, c, 1, g, g->dx);
        REAL DzmAtauxz = dbwd_p(mu, A->tauxz, c, Nx, g, g->dz);
        REAL DzpAtauz = dfwd_l2m(lam, mu, A->tauz, c, Nx, g, g->dz);
        REAL DzpAtaux = dfwd_p(lam, A->taux, c, Nx, g, g->dz);
        REAL DxpAtauxz = dfwd_p(mu, A->tauxz, c, 1, g, g->dx);
        A->vx[c] += -g->dt * ((2 * M->dxpml[c] + M->dzpml[c]) * A->vx[c] + (DxmAtaux + DxmAtauz + DzmAtauxz));
        A->vz[c] += -g->dt * ((M->dxpml[c] + 2 * M->dzpml[c]) * A->vz[c] + (DzpAtaux + DzpAtauz + DxpAtauxz));
    }
}

/* Test builds with IMG_ROUND set (REAL = float only) round the imaging's
 * five differences of the forward state to nearest even before use: 1 at
 * BF16 (8 mantissa bits), 2 at 24 bits (15 mantissa bits), as a store of
 * difference sets in those formats would.  IMG_ROUND 0 (the oracle) leaves
 * the expressions as they are. */
#ifndef IMG_ROUND
#define IMG_ROUND 0
#endif
#if IMG_ROUND
static inline float img_round(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    if (IMG_ROUND == 1) {
        u += 0x7FFFu + ((u >> 16) & 1u);
        u &= 0xFFFF0000u;
    } else {
        u += 0x7Fu + ((u >> 8) & 1u);
        u &= 0xFFFFFF00u;
    }
    memcpy(&x, &u, 4);
    return x;
}
#endif

/* ---- zero-lag imaging (elastic.cl:470-526) ------------------------------
 * G[0]=Gmu G[1]=Glam G[2]=Grho, G[3..5] the matching energy accumulators.
 * DzpVx is formed from vz, as in the reference (elastic.cl:485). */
void orc_grad(const orc_cfg *g, const orc_state *S, const orc_state *A, const orc_model *M, REAL *const *G)
{
    const long Nx = g->Nx, lo = g->npml + g->sdo;
    const double dt = g->dt;
#pragma omp parallel for schedule(static)
    for (long i = lo; i <= (long)g->Nz - g->sdo - g->npml; ++i)
        for (long j = lo; j <= (long)g->Nx - g->sdo - g->npml; ++j) {
            long c = i * Nx + j;
            REAL DzpVx = dfwd(S->vz, c, Nx, g, g->dz);
            REAL DxmVz = dbwd(S->vz, c, 1, g, g->dx);
            REAL DxpVx = dfwd(S->vx, c, 1, g, g->dx);
            REAL DzmVz = dbwd(S->vz, c, Nx, g, g->dz);
            REAL DzpPz = dfwd(S->tauz, c, Nx, g, g->dz);
            REAL DxmPx = dbwd(S->taux, c, 1, g, g->dx);
            REAL DxpPxz = dfwd(S->tauxz, c, 1, g, g->dx);
            REAL DzmPxz = dbwd(S->tauxz, c, Nx, g, g->dz);
#if IMG_ROUND
            /* the five imaged values rounded as a store of difference sets
             * would keep them (test builds only, see img_round) */
            DxpVx = img_round(DxpVx);
            DzmVz = img_round(DzmVz);
            const REAL q_vz = img_round(DzpVx + DxmVz), q_tx = img_round(DxmPx + DzmPxz), q_tz = img_round(DzpPz + DxpPxz);
#define Q_VZ q_vz
#define Q_TX q_tx
#define Q_TZ q_tz
#else
#define Q_VZ (DzpVx + DxmVz)
#define Q_TX (DxmPx + DzmPxz)
#define Q_TZ (DzpPz + DxpPxz)
#endif
            REAL tx = S->taux[c], tz = S->tauz[c], txz = S->tauxz[c], vx = S->vx[c], vz = S->vz[c];
            REAL rb = M->rho_b[c];
            G[0][c] += 2 * dt * (A->taux[c] * DxpVx + A->tauz[c] * DzmVz) + dt * A->tauxz[c] * Q_VZ;
            G[3][c] += 4 * dt * dt * (tx * tx * DxpVx * DxpVx + tz * tz * DzmVz * DzmVz) +
                       dt * dt * txz * txz * (DzpVx * DzpVx + DxmVz * DxmVz);
            G[1][c] += dt * (A->taux[c] + A->tauz[c]) * (DxpVx + DzmVz);
            G[4][c] += dt * dt * (tx * tx + tz * tz) * (DxpVx * DxpVx + DzmVz * DzmVz);
            G[2][c] += -(dt * (rb * rb)) * (A->vx[c] * Q_TX + A->vz[c] * Q_TZ);
#undef Q_VZ
#undef Q_TX
#undef Q_TZ
            G[5][c] += dt * dt * (vx * vx * (DxmPx * DxmPx + DzmPxz * DzmPxz) + vz * vz * (DzpPz * DzpPz + DxpPxz * DxpPxz));
        }
}

/* ---- per-shot drivers ----------------------------------------------------
 * Guarded scratch: every field gets GUARD zero elements on each side. */
static long guard_of(const orc_cfg *g) { return 4L * g->Nx + 8; }

static REAL *galloc(const orc_cfg *g, REAL **base)
{
    long n = (long)g->Nz * g->Nx, gd = guard_of(g);
    *base = (REAL *)calloc((size_t)(n + 2 * gd), sizeof(REAL));
    return *base ? *base + gd : NULL;
}

typedef struct {
    REAL *base[5];
    orc_state s;
} gstate;

static int gstate_new(const orc_cfg *g, gstate *st)
{
    REAL **p[5] = {&st->s.vx, &st->s.vz, &st->s.taux, &st->s.tauz, &st->s.tauxz};
    for (int k = 0; k < 5; ++k) {
        *p[k] = galloc(g, &st->base[k]);
        if (!*p[k]) return -1;
    }
    return 0;
}

static void gstate_free(gstate *st)
{
    for (int k = 0; k < 5; ++k) free(st->base[k]);
}

static void state_save(const orc_cfg *g, const orc_state *S, REAL *dst /* [5][Nz*Nx] */)
{
    long n = (long)g->Nz * g->Nx;
    const REAL *f[5] = {S->vx, S->vz, S->taux, S->tauz, S->tauxz};
    for (int k = 0; k < 5; ++k) memcpy(dst + k * n, f[k], (size_t)n * sizeof(REAL));
}

static void state_load(const orc_cfg *g, orc_state *S, const REAL *src)
{
    long n = (long)g->Nz * g->Nx;
    REAL *f[5] = {S->vx, S->vz, S->taux, S->tauz, S->tauxz};
    for (int k = 0; k < 5; ++k) memcpy(f[k], src + k * n, (size_t)n * sizeof(REAL));
}

/* Model arrays are copied into guarded storage so stencils may read past
 * the array ends. */
typedef struct {
    REAL *base[5];
    orc_model m;
} gmodel;

static int gmodel_new(const orc_cfg *g, gmodel *gm, const REAL *lam, const REAL *mu, const REAL *rho_b,
                      const REAL *dxpml, const REAL *dzpml)
{
    const REAL *src[5] = {lam, mu, rho_b, dxpml, dzpml};
    REAL *dst[5];
    long n = (long)g->Nz * g->Nx;
    for (int k = 0; k < 5; ++k) {
        dst[k] = galloc(g, &gm->base[k]);
        if (!dst[k]) return -1;
        memcpy(dst[k], src[k], (size_t)n * sizeof(REAL));
    }
    gm->m.lam = dst[0];
    gm->m.mu = dst[1];
    gm->m.rho_b = dst[2];
    gm->m.dxpml = dst[3];
    gm->m.dzpml = dst[4];
    return 0;
}

static void gmodel_free(gmodel *gm)
{
    for (int k = 0; k < 5; ++k) free(gm->base[k]);
}

static void step_forward(const orc_cfg *g, orc_state *S, const orc_model *M, int coeff)
{
    /* order of WavePropagator.__update_fwd, wave_propagation.py:666-697 */
    orc_update_velx(g, coeff, S, M);
    orc_update_velz(g, coeff, S, M);
    orc_update_tauz(g, coeff, S, M);
    orc_update_tauxz(g, coeff, S, M);
}

static void step_reverse(const orc_cfg *g, orc_state *S, const orc_model *M)
{
    /* reverse-time reconstruction order, wave_propagation.py:782-812 */
    orc_update_tauxz(g, -1, S, M);
    orc_update_tauz(g, -1, S, M);
    orc_update_velz(g, -1, S, M);
    orc_update_velx(g, -1, S, M);
}

static int in_list(const int32_t *a, int n, int v)
{
    for (int k = 0; k < n; ++k)
        if (a[k] == v) return 1;
    return 0;
}

/* One shot of WavePropagator.__kernel (wave_propagation.py:699-733).
 * src_vals[n_inj][4] holds the wavelet sample times the source component for
 * (vx, vz, taux, tauz) at each injection index.  seis[5][nt_ext][Nr] is
 * written for this shot; W (nullable) receives the state after every step in
 * chp: W[k][5][Nz*Nx].  Returns 0, or -1 on allocation failure. */
int orc_forward_shot(const orc_cfg *g, const REAL *lam, const REAL *mu, const REAL *rho_b, const REAL *dxpml,
                     const REAL *dzpml, int32_t srcx, int32_t srcz, const float *src_vals, int32_t n_src_vals,
                     REAL *seis, REAL *W, const int32_t *chp, int32_t nchp)
{
    gstate st;
    gmodel gm;
    memset(&st, 0, sizeof st);
    memset(&gm, 0, sizeof gm);
    if (gstate_new(g, &st) || gmodel_new(g, &gm, lam, mu, rho_b, dxpml, dzpml)) {
        gstate_free(&st);
        gmodel_free(&gm);
        return -1;
    }
    const long n5 = 5L * g->Nz * g->Nx;
    long t_src = 0, chpc = 0;
    const float zero4[4] = {0, 0, 0, 0};
    for (long t = 0; t < g->nt; ++t) {
        if (t % g->dt_scale == 0) {
            orc_record(g, &st.s, seis, t_src);
            orc_add_source(g, &st.s, srcx, srcz, t_src < n_src_vals ? src_vals + 4 * t_src : zero4);
            t_src += 1;
        }
        step_forward(g, &st.s, &gm.m, +1);
        if (W && in_list(chp, nchp, (int)t)) {
            state_save(g, &st.s, W + chpc * n5);
            chpc += 1;
        }
    }
    gstate_free(&st);
    gmodel_free(&gm);
    return 0;
}

/* One shot of WavePropagator.__kernel_gradient (wave_propagation.py:751-856).
 * res[5] point at this shot's residual planes [nt_ext][Nr] (NULL = zero
 * component).  W holds the states the forward pass stored at chp.  G[6]
 * accumulate (Gmu, Glam, Grho, and the three energy terms) over shots. */
int orc_gradient_shot(const orc_cfg *g, const REAL *lam, const REAL *mu, const REAL *rho_b, const REAL *dxpml,
                      const REAL *dzpml, const REAL *const *res, const REAL *W, const int32_t *chp, int32_t nchp,
                      REAL *G0, REAL *G1, REAL *G2, REAL *G3, REAL *G4, REAL *G5)
{
    gstate fw, ad;
    gmodel gm;
    memset(&fw, 0, sizeof fw);
    memset(&ad, 0, sizeof ad);
    memset(&gm, 0, sizeof gm);
    if (gstate_new(g, &fw) || gstate_new(g, &ad) || gmodel_new(g, &gm, lam, mu, rho_b, dxpml, dzpml)) {
        gstate_free(&fw);
        gstate_free(&ad);
        gmodel_free(&gm);
        return -1;
    }
    REAL *const G[6] = {G0, G1, G2, G3, G4, G5};
    const long n5 = 5L * g->Nz * g->Nx;
    long chpc = nchp - 1, t_src = g->nt_ext;
    for (long t = g->nt - 1; t > 0; --t) {
        /* python indexing: chp[-1] is the last element */
        long k = chpc >= 0 ? chpc : chpc + nchp;
        if (t == chp[k]) {
            state_load(g, &fw.s, W + k * n5);
            chpc -= 1;
        } else {
            step_reverse(g, &fw.s, &gm.m);
        }
        if (t % g->dt_scale == 0) {
            long row = t_src - 1;
            if (row < 0) row += g->nt_ext; /* numpy negative index */
            const REAL *r[5];
            for (int c = 0; c < 5; ++c) r[c] = res[c] ? res[c] + row * (long)g->Nr : NULL;
            orc_adj_inject(g, &ad.s, r);
            t_src -= 1;
        }
        orc_adj_update_tau(g, &ad.s, &gm.m);
        orc_adj_update_v(g, &ad.s, &gm.m);
        orc_grad(g, &fw.s, &ad.s, &gm.m, G);
    }
    gstate_free(&fw);
    gstate_free(&ad);
    gmodel_free(&gm);
    return 0;
}

/* ---- exact discrete adjoint (no counterpart in the reference) -----------
 * The transpose of one forward step of this file (record, source add,
 * velocity update + damping, stress update + damping, each on the update
 * domain), so that the gradient it accumulates is the exact derivative of
 * J = 1/2 sum (traces - observed)^2 with respect to lam, mu and the
 * buoyancy b on the padded grid, the damping profiles held fixed.  The
 * transposed differences use (D+)^T = -D- and (D-)^T = -D+ on fields that
 * are zero outside the update domain; cells outside the grid read as zero
 * (no flat-index wrap, which only ever reaches constant zero cells in the
 * forward step). */
static inline double at0(const REAL *f, const orc_cfg *g, long i, long j)
{
    return (i < 0 || i >= g->Nz || j < 0 || j >= g->Nx) ? 0.0 : (double)f[i * g->Nx + j];
}

static double sfwd(const REAL *f, const orc_cfg *g, long i, long j, int di, int dj, double h)
{
    const double c[4] = {g->c1, g->c2, g->c3, g->c4};
    double s = 0.0;
    for (int q = 0; q < 4; ++q)
        s += c[q] * (at0(f, g, i + (q + 1) * di, j + (q + 1) * dj) - at0(f, g, i - q * di, j - q * dj));
    return s / h;
}

static double sbwd(const REAL *f, const orc_cfg *g, long i, long j, int di, int dj, double h)
{
    const double c[4] = {g->c1, g->c2, g->c3, g->c4};
    double s = 0.0;
    for (int q = 0; q < 4; ++q)
        s += c[q] * (at0(f, g, i + q * di, j + q * dj) - at0(f, g, i - (q + 1) * di, j - (q + 1) * dj));
    return s / h;
}

static inline int in_dom(const orc_cfg *g, long i, long j)
{
    return i >= g->sdo && i <= (long)g->Nz - g->sdo && j >= g->sdo && j <= (long)g->Nx - g->sdo;
}

/* Transpose of orc_record for one trace row: add the residual of every trace
 * slot to the adjoint of the field it recorded (the crosswell vz trace holds
 * vx, elastic_crosswell.cl:27). */
static inline void radj5(const orc_cfg *g, orc_state *A, const REAL *const *res, long ir, long cell, int vz_from_vx)
{
    REAL *f[5] = {A->vx, vz_from_vx ? A->vx : A->vz, A->taux, A->tauz, A->tauxz};
    if (ir < 0 || ir >= g->Nr || cell < 0 || cell >= (long)g->Nz * g->Nx) return;
    for (int k = 0; k < 5; ++k)
        if (res[k]) f[k][cell] += res[k][ir];
}

static void record_adjoint(const orc_cfg *g, orc_state *A, const REAL *const *res)
{
    const long Nx = g->Nx, Nz = g->Nz;
    if (g->acq_type == 1 || g->acq_type == 2) {
        long i = g->rec_surface_const;
        long off = (g->acq_type == 2) ? g->n_extera_rec : 0;
        if (i >= 0 && i < Nz)
            for (long j = 0; j < Nx; j += g->dxr) {
                long ir = j / g->dxr;
                if (ir < g->n_main_rec) radj5(g, A, res, off + ir, i * Nx + (j + g->rec_surface_var), 0);
            }
    }
    if (g->acq_type == 0) {
        long j = g->rec_top_right_const;
        if (j >= 0 && j < Nx)
            for (long i = 0; i < Nz; i += g->dxr) radj5(g, A, res, i / g->dxr, (i + g->rec_top_right_var) * Nx + j, 1);
    }
    if (g->acq_type == 2) {
        long j = g->rec_top_left_const;
        if (j >= 0 && j < Nx)
            for (long i = 0; i < Nz; i += g->dxr) {
                long ir = i / g->dxr;
                if (ir < g->n_extera_rec) radj5(g, A, res, ir, (i + g->rec_top_left_var) * Nx + j, 0);
            }
        j = g->rec_top_right_const;
        long start = g->n_extera_rec + g->n_main_rec;
        if (j >= 0 && j < Nx)
            for (long i = 0; i < Nz; i += g->dxr)
                radj5(g, A, res, start + i / g->dxr, (i + g->rec_top_right_var) * Nx + j, 0);
    }
}

/* One shot.  W[t] (t = 0 .. nt-1) is the state after step t, S_{t+1}; S_0 is
 * zero.  res[5]: this shot's dJ/dtrace planes [nt_ext][Nr] (NULL = zero).
 * Accumulates dJ/dlam, dJ/dmu, dJ/db on the padded grid into Glam, Gmu, Gb. */
int orc_exact_gradient_shot(const orc_cfg *g, const REAL *lam, const REAL *mu, const REAL *rho_b, const REAL *dxpml,
                            const REAL *dzpml, int32_t srcx, int32_t srcz, const float *src_vals, int32_t n_src_vals,
                            const REAL *const *res, const REAL *W, REAL *Glam, REAL *Gmu, REAL *Gb)
{
    const long Nz = g->Nz, Nx = g->Nx, n = Nz * Nx, n5 = 5 * n;
    const double dt = g->dt;
    REAL *buf = (REAL *)calloc((size_t)(5 + 5 + 5) * n, sizeof(REAL));
    if (!buf) return -1;
    REAL *L = buf;            /* adjoint state, [5][n] */
    REAL *P = buf + 5 * n;    /* P1, P2, P3, Q1, Q2 */
    REAL *S0 = buf + 10 * n;  /* S_t with the source added */
    orc_state A = {L, L + n, L + 2 * n, L + 3 * n, L + 4 * n};
    REAL *P1 = P, *P2 = P + n, *P3 = P + 2 * n, *Q1 = P + 3 * n, *Q2 = P + 4 * n;
    for (long t = g->nt - 1; t >= 0; --t) {
        const REAL *S1 = W + t * n5;
        if (t > 0)
            memcpy(S0, W + (t - 1) * n5, (size_t)n5 * sizeof(REAL));
        else
            memset(S0, 0, (size_t)n5 * sizeof(REAL));
        if (t % g->dt_scale == 0 && srcz >= 0 && srcz < Nz && srcx >= 0 && srcx < Nx) {
            long k = t / g->dt_scale, c = (long)srcz * Nx + srcx;
            if (k < n_src_vals)
                for (int f = 0; f < 4; ++f) S0[f * n + c] += src_vals[4 * k + f];
        }
        const REAL *vx2 = S1, *vz2 = S1 + n, *txx0 = S0 + 2 * n, *tzz0 = S0 + 3 * n, *txz0 = S0 + 4 * n;
        /* stress update, transposed: P fields and the lam / mu gradient */
#pragma omp parallel for schedule(static)
        for (long i = 0; i < Nz; ++i)
            for (long j = 0; j < Nx; ++j) {
                long c = i * Nx + j;
                P1[c] = P2[c] = P3[c] = 0;
                if (!in_dom(g, i, j)) continue;
                double damp = 1.0 - dt * ((double)dxpml[c] + (double)dzpml[c]);
                double axx = damp * A.taux[c], azz = damp * A.tauz[c], axz = damp * A.tauxz[c];
                double l = lam[c], m = mu[c];
                P1[c] = (REAL)(dt * ((l + 2 * m) * axx + l * azz));
                P2[c] = (REAL)(dt * m * axz);
                P3[c] = (REAL)(dt * (l * axx + (l + 2 * m) * azz));
                double dxp_vx = sfwd(vx2, g, i, j, 0, 1, g->dx), dzm_vz = sbwd(vz2, g, i, j, 1, 0, g->dz);
                double dxm_vz = sbwd(vz2, g, i, j, 0, 1, g->dx), dzp_vx = sfwd(vx2, g, i, j, 1, 0, g->dz);
                Glam[c] += (REAL)(dt * (axx + azz) * (dxp_vx + dzm_vz));
                Gmu[c] += (REAL)(dt * (2 * axx * dxp_vx + 2 * azz * dzm_vz + axz * (dxm_vz + dzp_vx)));
                A.taux[c] = (REAL)axx;
                A.tauz[c] = (REAL)azz;
                A.tauxz[c] = (REAL)axz;
            }
        /* velocity update, transposed: Q fields and the buoyancy gradient */
#pragma omp parallel for schedule(static)
        for (long i = 0; i < Nz; ++i)
            for (long j = 0; j < Nx; ++j) {
                long c = i * Nx + j;
                double mvx = A.vx[c] - sbwd(P1, g, i, j, 0, 1, g->dx) - sbwd(P2, g, i, j, 1, 0, g->dz);
                double mvz = A.vz[c] - sfwd(P3, g, i, j, 1, 0, g->dz) - sfwd(P2, g, i, j, 0, 1, g->dx);
                Q1[c] = Q2[c] = 0;
                if (in_dom(g, i, j)) {
                    double damp = 1.0 - dt * ((double)dxpml[c] + (double)dzpml[c]);
                    double bx = damp * mvx, bz = damp * mvz, b = rho_b[c];
                    Q1[c] = (REAL)(dt * b * bx);
                    Q2[c] = (REAL)(dt * b * bz);
                    Gb[c] += (REAL)(dt * (bx * (sbwd(txx0, g, i, j, 0, 1, g->dx) + sbwd(txz0, g, i, j, 1, 0, g->dz)) +
                                          bz * (sfwd(tzz0, g, i, j, 1, 0, g->dz) + sfwd(txz0, g, i, j, 0, 1, g->dx))));
                    mvx = bx;
                    mvz = bz;
                }
                S0[c] = (REAL)mvx; /* S0's vx / vz planes are free scratch now */
                S0[n + c] = (REAL)mvz;
            }
        memcpy(A.vx, S0, (size_t)n * sizeof(REAL));
        memcpy(A.vz, S0 + n, (size_t)n * sizeof(REAL));
#pragma omp parallel for schedule(static)
        for (long i = 0; i < Nz; ++i)
            for (long j = 0; j < Nx; ++j) {
                long c = i * Nx + j;
                A.taux[c] = (REAL)(A.taux[c] - sfwd(Q1, g, i, j, 0, 1, g->dx));
                A.tauz[c] = (REAL)(A.tauz[c] - sbwd(Q2, g, i, j, 1, 0, g->dz));
                A.tauxz[c] = (REAL)(A.tauxz[c] - sfwd(Q1, g, i, j, 1, 0, g->dz) - sbwd(Q2, g, i, j, 0, 1, g->dx));
            }
        if (t % g->dt_scale == 0 && t / g->dt_scale < g->nt_ext) {
            const REAL *r[5];
            for (int c = 0; c < 5; ++c) r[c] = res[c] ? res[c] + (t / g->dt_scale) * (long)g->Nr : NULL;
            record_adjoint(g, &A, r);
        }
    }
    free(buf);
    return 0;
}

/* Single-kernel entry points on caller-guarded arrays, for unit checks of one
 * step against the product's kernels. */
void orc_step_forward(const orc_cfg *g, REAL *vx, REAL *vz, REAL *taux, REAL *tauz, REAL *tauxz, const REAL *lam,
                      const REAL *mu, const REAL *rho_b, const REAL *dxpml, const REAL *dzpml, int coeff)
{
    orc_state S = {vx, vz, taux, tauz, tauxz};
    orc_model M = {lam, mu, rho_b, dxpml, dzpml};
    if (coeff == 1)
        step_forward(g, &S, &M, 1);
    else
        step_reverse(g, &S, &M);
}

int orc_sizeof_real(void) { return (int)sizeof(REAL); }
