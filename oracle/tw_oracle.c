/*
 * tw_oracle.c -- FP64 CPU restatement of TeraWarp's warp path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file; it is the checker that the CUDA path is compared against
 * (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * legs are its only users).
 *
 * PARITY STATUS: unpinned.  The reference (TCloudd/TeraWarp) ships no tests,
 * fixtures or golden vectors, and its CPU path cannot be compiled here: it
 * needs Qt4, Vaa3D basic_c_fun and newmat11 (plugin_Bigimagewarp.pro:2-36),
 * none of which is present.  This file therefore restates the reference's own
 * arithmetic line by line (citations below, paths relative to the reference
 * project) and is pinned only by project-written known-answer tests
 * (identity, pure affine, B-spline reproduction, integer shifts, OOB -> 0)
 * and by an independent numpy/scipy solve of the same TPS system.
 *
 * Conventions copied from the reference:
 *   - volumes are x-fastest, then y, z, channel  (basic_memory.cpp:148-168)
 *   - both warps are pull-back: every output voxel p samples the subject at q(p)
 *   - TPS: q = p + DF(p); out = (T)(trilinear + 0.5)   (q_imgwarp_tps_quicksmallmemory.cpp:85-167)
 *   - affine: q = M [x y z 1]^T; out = (T)(trilinear)   (q_warp_affine_tps.cpp:1373-1437)
 *   - a sample with any q_i < 0 or q_i > sz_i - 1 writes 0
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_OK 0
#define OR_ERR_ARG 1
#define OR_ERR_SINGULAR 2
#define OR_ERR_OOM 3

static void set_threads(int threads)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

int or_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_num_procs();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* Dense FP64 helpers (row-major).                                           */
/* ------------------------------------------------------------------------- */

/* Householder QR of the n x 4 matrix X (row-major, overwritten).  Produces the
 * thin orthonormal factor Qt (n x 4) and the upper-triangular R (4 x 4) with
 * X = Qt R.  Stands in for newmat's QRZ(X, R) at
 * q_imgwarp_tps_quicksmallmemory.cpp:571; the sign convention of the factors
 * does not reach c or d (c = q2 A^-1 q2' Y is invariant to the basis of q2,
 * and r^-1 q1' is the pseudo-inverse of X). */
static int householder_qr_n4(int n, double *X, double *Qt, double *R)
{
    double *V = (double *)calloc((size_t)n * 4, sizeof(double));
    double tau[4];
    if (!V) return OR_ERR_OOM;
    for (int k = 0; k < 4; ++k) {
        double nrm = 0.0;
        for (int i = k; i < n; ++i) nrm += X[(size_t)i * 4 + k] * X[(size_t)i * 4 + k];
        nrm = sqrt(nrm);
        double alpha = X[(size_t)k * 4 + k] > 0 ? -nrm : nrm;
        for (int i = 0; i < n; ++i) V[(size_t)i * 4 + k] = (i < k) ? 0.0 : X[(size_t)i * 4 + k];
        V[(size_t)k * 4 + k] -= alpha;
        double vv = 0.0;
        for (int i = k; i < n; ++i) vv += V[(size_t)i * 4 + k] * V[(size_t)i * 4 + k];
        tau[k] = vv > 0 ? 2.0 / vv : 0.0;
        for (int j = k; j < 4; ++j) {
            double s = 0.0;
            for (int i = k; i < n; ++i) s += V[(size_t)i * 4 + k] * X[(size_t)i * 4 + j];
            s *= tau[k];
            for (int i = k; i < n; ++i) X[(size_t)i * 4 + j] -= s * V[(size_t)i * 4 + k];
        }
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) R[i * 4 + j] = (j >= i) ? X[(size_t)i * 4 + j] : 0.0;
    /* Qt = H1 H2 H3 H4 [I4; 0] */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < 4; ++j) Qt[(size_t)i * 4 + j] = (i == j) ? 1.0 : 0.0;
    for (int k = 3; k >= 0; --k) {
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int i = k; i < n; ++i) s += V[(size_t)i * 4 + k] * Qt[(size_t)i * 4 + j];
            s *= tau[k];
            for (int i = k; i < n; ++i) Qt[(size_t)i * 4 + j] -= s * V[(size_t)i * 4 + k];
        }
    }
    free(V);
    for (int i = 0; i < 4; ++i)
        if (fabs(R[i * 4 + i]) < 1e-9 * (1.0 + fabs(R[0]))) return OR_ERR_SINGULAR;
    return OR_OK;
}

/* LU with partial pivoting, in place (n x n row-major); solves A x = b for
 * nrhs right-hand sides stored row-major n x nrhs in B.  Stands in for
 * newmat's A.i() at q_imgwarp_tps_quicksmallmemory.cpp:582. */
static int lu_solve(int n, double *A, int nrhs, double *B)
{
    int *piv = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!piv) return OR_ERR_OOM;
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; ++i) {
            double v = fabs(A[(size_t)i * n + k]);
            if (v > best) { best = v; p = i; }
        }
        if (best == 0.0) { free(piv); return OR_ERR_SINGULAR; }
        piv[k] = p;
        if (p != k) {
            for (int j = 0; j < n; ++j) {
                double t = A[(size_t)k * n + j]; A[(size_t)k * n + j] = A[(size_t)p * n + j]; A[(size_t)p * n + j] = t;
            }
            for (int j = 0; j < nrhs; ++j) {
                double t = B[(size_t)k * nrhs + j]; B[(size_t)k * nrhs + j] = B[(size_t)p * nrhs + j]; B[(size_t)p * nrhs + j] = t;
            }
        }
        double inv = 1.0 / A[(size_t)k * n + k];
#pragma omp parallel for schedule(static)
        for (int i = k + 1; i < n; ++i) {
            double f = A[(size_t)i * n + k] * inv;
            A[(size_t)i * n + k] = f;
            double *ri = A + (size_t)i * n;
            const double *rk = A + (size_t)k * n;
            for (int j = k + 1; j < n; ++j) ri[j] -= f * rk[j];
            for (int j = 0; j < nrhs; ++j) B[(size_t)i * nrhs + j] -= f * B[(size_t)k * nrhs + j];
        }
    }
    for (int k = n - 1; k >= 0; --k) {
        for (int j = 0; j < nrhs; ++j) {
            double s = B[(size_t)k * nrhs + j];
            for (int i = k + 1; i < n; ++i) s -= A[(size_t)k * n + i] * B[(size_t)i * nrhs + j];
            B[(size_t)k * nrhs + j] = s / A[(size_t)k * n + k];
        }
    }
    free(piv);
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* (a-1) TPS solve                                                            */
/* ------------------------------------------------------------------------- */

/* Restates compute_df_stps_subsampled_volume_4bspline's CPU branch
 * (q_imgwarp_tps_quicksmallmemory.cpp:377-444 and :554-586; identical in the
 * tiled _per variant :906-1082):
 *
 *   K(i,j) = -|s_i - s_j|                       (:437-444, from float coords)
 *   X = [1 s], Y = [1 t]                        (:559-569)
 *   X = Q R (QRZ), extend_orthonormal(Q, 4)     (:570-573; algorithm visible
 *                                                in extendornormal.cu:85-127)
 *   q1 = Q(:,1:4), q2 = Q(:,5:n), r = R(1:4,1:4)
 *   A  = q2' K q2 + lambda I                    (:580, lambda = 0.2)
 *   c  = q2 (A^-1 q2' Y)                        (:581)
 *   d  = r^-1 q1' (Y - K c)                     (:583)
 *
 * ctr = TPS centres (the function's "matchSubjectPos"), val = values
 * ("matchTargetPos"), both n x 3 float.  c is n x 4 row-major, d is 4 x 4
 * row-major.  f(p) = [1 p] d + sum_n -|p - s_n| c_n. */
int or_tps_solve(int n, const float *ctr, const float *val, double lambda, int threads,
                 double *c_out, double *d_out)
{
    if (n < 4 || !ctr || !val || !c_out || !d_out) return OR_ERR_ARG;
    set_threads(threads);
    const int m = n - 4;
    int rc = OR_OK;
    double *K = (double *)malloc(sizeof(double) * (size_t)n * n);
    double *X = (double *)malloc(sizeof(double) * (size_t)n * 4);
    double *Y = (double *)malloc(sizeof(double) * (size_t)n * 4);
    double *Q = (double *)calloc((size_t)n * n, sizeof(double)); /* row-major n x n */
    double *Qt = (double *)malloc(sizeof(double) * (size_t)n * 4);
    double *SSR = (double *)calloc((size_t)n, sizeof(double));
    double *col = (double *)malloc(sizeof(double) * (size_t)n);
    double R[16];
    double *KQ = NULL, *A = NULL, *Z = NULL;
    if (!K || !X || !Y || !Q || !Qt || !SSR || !col) { rc = OR_ERR_OOM; goto done; }

#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) {
            double dx = (double)ctr[3 * i + 0] - (double)ctr[3 * j + 0];
            double dy = (double)ctr[3 * i + 1] - (double)ctr[3 * j + 1];
            double dz = (double)ctr[3 * i + 2] - (double)ctr[3 * j + 2];
            K[(size_t)i * n + j] = -sqrt(dx * dx + dy * dy + dz * dz);
        }
    }
    for (int i = 0; i < n; ++i) {
        X[i * 4 + 0] = 1.0;
        X[i * 4 + 1] = ctr[3 * i + 0];
        X[i * 4 + 2] = ctr[3 * i + 1];
        X[i * 4 + 3] = ctr[3 * i + 2];
        Y[i * 4 + 0] = 1.0;
        Y[i * 4 + 1] = val[3 * i + 0];
        Y[i * 4 + 2] = val[3 * i + 1];
        Y[i * 4 + 3] = val[3 * i + 2];
    }
    rc = householder_qr_n4(n, X, Qt, R);
    if (rc) goto done;

    /* extend_orthonormal(Q, 4): complete Q to an n x n orthonormal basis by
     * Gram-Schmidt on unit vectors e_k, always picking the row k whose
     * current sum of squares is smallest (extendornormal.cu:85-127). */
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < 4; ++j) {
            Q[(size_t)i * n + j] = Qt[(size_t)i * 4 + j];
            SSR[i] += Qt[(size_t)i * 4 + j] * Qt[(size_t)i * 4 + j];
        }
    }
    for (int i = 4; i < n; ++i) {
        int k = 0;
        double mn = SSR[0];
        for (int r = 1; r < n; ++r)
            if (SSR[r] < mn) { mn = SSR[r]; k = r; }
        const double *qk = Q + (size_t)k * n;
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; ++r) {
            const double *qr = Q + (size_t)r * n;
            double s = 0.0;
            for (int j = 0; j < i; ++j) s += -qr[j] * qk[j];
            col[r] = s;
        }
        col[k] += 1.0;
        double ss = 0.0;
        for (int r = 0; r < n; ++r) ss += col[r] * col[r];
        ss = sqrt(ss);
        for (int r = 0; r < n; ++r) {
            col[r] /= ss;
            SSR[r] += col[r] * col[r];
            Q[(size_t)r * n + i] = col[r];
        }
    }

    /* A = q2' K q2 + lambda I, with KQ = K q2 (n x m) */
    KQ = (double *)malloc(sizeof(double) * (size_t)n * (m > 0 ? m : 1));
    A = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1) * (m > 0 ? m : 1));
    Z = (double *)calloc((size_t)(m > 0 ? m : 1) * 4, sizeof(double));
    if (!KQ || !A || !Z) { rc = OR_ERR_OOM; goto done; }
    if (m > 0) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            double *out = KQ + (size_t)i * m;
            for (int j = 0; j < m; ++j) out[j] = 0.0;
            const double *ki = K + (size_t)i * n;
            for (int l = 0; l < n; ++l) {
                const double kil = ki[l];
                const double *ql = Q + (size_t)l * n + 4;
                for (int j = 0; j < m; ++j) out[j] += kil * ql[j];
            }
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < m; ++i) {
            double *out = A + (size_t)i * m;
            for (int j = 0; j < m; ++j) out[j] = 0.0;
            for (int l = 0; l < n; ++l) {
                const double qli = Q[(size_t)l * n + 4 + i];
                const double *kl = KQ + (size_t)l * m;
                for (int j = 0; j < m; ++j) out[j] += qli * kl[j];
            }
            out[i] += lambda;
        }
        /* Z = q2' Y (m x 4) */
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < 4; ++j) {
                double s = 0.0;
                for (int l = 0; l < n; ++l) s += Q[(size_t)l * n + 4 + i] * Y[(size_t)l * 4 + j];
                Z[(size_t)i * 4 + j] = s;
            }
        rc = lu_solve(m, A, 4, Z);
        if (rc) goto done;
    }
    /* c = q2 Z */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int l = 0; l < m; ++l) s += Q[(size_t)i * n + 4 + l] * Z[(size_t)l * 4 + j];
            c_out[(size_t)i * 4 + j] = s;
        }
    /* d = r^-1 q1' (Y - K c) */
    {
        double W[16] = {0};
        for (int i = 0; i < n; ++i) {
            double res[4];
            for (int j = 0; j < 4; ++j) {
                double s = 0.0;
                for (int l = 0; l < n; ++l) s += K[(size_t)i * n + l] * c_out[(size_t)l * 4 + j];
                res[j] = Y[(size_t)i * 4 + j] - s;
            }
            for (int a = 0; a < 4; ++a)
                for (int j = 0; j < 4; ++j) W[a * 4 + j] += Q[(size_t)i * n + a] * res[j];
        }
        for (int j = 0; j < 4; ++j) {
            for (int a = 3; a >= 0; --a) {
                double s = W[a * 4 + j];
                for (int b = a + 1; b < 4; ++b) s -= R[a * 4 + b] * d_out[b * 4 + j];
                d_out[a * 4 + j] = s / R[a * 4 + a];
            }
        }
    }
done:
    free(K); free(X); free(Y); free(Q); free(Qt); free(SSR); free(col);
    free(KQ); free(A); free(Z);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* (a-2) TPS evaluation at the coarse control-grid nodes                     */
/* ------------------------------------------------------------------------- */

/* Grid size rule gsz = ceil(sz/g) + 1 + 2 (q_imgwarp_tps_quicksmallmemory.cpp:592,1090). */
int64_t or_grid_size(int64_t sz, int g)
{
    return (int64_t)ceil((double)sz / (double)g) + 1 + 2;
}

/* Node (i,j,k) sits at ((i-1)g+ox, (j-1)g+oy, (k-1)g+oz); its displacement is
 * f(p) - p with f(p) = [1 p] d + sum_n -|p - s_n| c_n, accumulated in double
 * in landmark order and stored as float (DisplaceFieldF3D, q_littleQuickWarp_common.h:50-55).
 * Restates q_imgwarp_tps_quicksmallmemory.cpp:620-648 (serial whole image)
 * and :1117-1146 (OpenMP over z, tiles with offsets).  df is gsz2 x gsz1 x
 * gsz0 x 3 floats (x fastest, component innermost). */
int or_tps_grid(int n, const float *ctr, const double *c, const double *d,
                int64_t gsz0, int64_t gsz1, int64_t gsz2, int g,
                int64_t ox, int64_t oy, int64_t oz, int threads, float *df)
{
    if (n < 1 || g < 1 || gsz0 < 1 || gsz1 < 1 || gsz2 < 1 || !df) return OR_ERR_ARG;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) if (threads != 1)
    for (int64_t k = 0; k < gsz2; ++k) {
        for (int64_t j = 0; j < gsz1; ++j) {
            for (int64_t i = 0; i < gsz0; ++i) {
                double px = (double)((i - 1) * g + ox);
                double py = (double)((j - 1) * g + oy);
                double pz = (double)((k - 1) * g + oz);
                double xo[4] = {1.0, px, py, pz};
                double fa[4], fk[4] = {0, 0, 0, 0};
                for (int col = 0; col < 4; ++col) {
                    double s = 0.0;
                    for (int r = 0; r < 4; ++r) s += xo[r] * d[r * 4 + col];
                    fa[col] = s;
                }
                for (int nn = 0; nn < n; ++nn) {
                    double dx = px - (double)ctr[3 * nn + 0];
                    double dy = py - (double)ctr[3 * nn + 1];
                    double dz = pz - (double)ctr[3 * nn + 2];
                    double kv = -sqrt(dx * dx + dy * dy + dz * dz);
                    for (int col = 0; col < 4; ++col) fk[col] += kv * c[(size_t)nn * 4 + col];
                }
                float *o = df + 3 * (size_t)((k * gsz1 + j) * gsz0 + i);
                o[0] = (float)(fa[1] + fk[1] - px);
                o[1] = (float)(fa[2] + fk[2] - py);
                o[2] = (float)(fa[3] + fk[3] - pz);
            }
        }
    }
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* (a-3) cubic B-spline basis and per-cell expansion                          */
/* ------------------------------------------------------------------------- */

/* q_nonrigid_ini_bsplinebasis_3D (q_imgwarp_tps_quicksmallmemory.cpp:663-699):
 * T(i,:) = [t^3 t^2 t 1] with t = i/n, TB = T B/6, and the n^3 x 64
 * Kronecker basis KP(KP(TB,TB),TB).  Only TB (n x 4) is returned; the
 * Kronecker entries are formed on the fly as (TB[i1][j1]*TB[i2][j2])*TB[i3][j3]
 * exactly as KP would compute them. */
int or_bspline_tb(int n, double *TB)
{
    if (n <= 0 || !TB) return OR_ERR_ARG;
    static const double Bi[4][4] = {{-1, 3, -3, 1}, {3, -6, 3, 0}, {-3, 0, 3, 0}, {1, 4, 1, 0}};
    double B[4][4];
    for (int r = 0; r < 4; ++r)
        for (int s = 0; s < 4; ++s) B[r][s] = Bi[r][s] / 6.0;
    double t_step = 1.0 / n;
    for (int i = 0; i < n; ++i) {
        double t = t_step * i;
        double T[4];
        for (int j = 0; j <= 3; ++j) T[j] = pow(t, 3 - j);
        for (int s = 0; s < 4; ++s) {
            double acc = 0.0;
            for (int r = 0; r < 4; ++r) acc += T[r] * B[r][s];
            TB[i * 4 + s] = acc;
        }
    }
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* (a-4) trilinear / nearest-neighbour sample                                 */
/* ------------------------------------------------------------------------- */

#define VOX(src, dt, idx) ((dt) == 1 ? (double)((const uint8_t *)(src))[(idx)] : (double)((const uint16_t *)(src))[(idx)])

/* Trilinear sample with the reference's floor/ceil weights
 * (q_imgwarp_tps_quicksmallmemory.cpp:132-160, q_warp_affine_tps.cpp:1401-1433).
 * Returns the un-rounded value; the caller applies +0.5 (TPS) or truncation (affine). */
static inline double trilinear(const void *src, int dt, int64_t sx, int64_t sy, const double *q)
{
    int64_t x_s = (int64_t)floor(q[0]), x_b = (int64_t)ceil(q[0]);
    int64_t y_s = (int64_t)floor(q[1]), y_b = (int64_t)ceil(q[1]);
    int64_t z_s = (int64_t)floor(q[2]), z_b = (int64_t)ceil(q[2]);
    double l_w = 1.0 - (q[0] - x_s), r_w = 1.0 - l_w;
    double t_w = 1.0 - (q[1] - y_s), b_w = 1.0 - t_w;
    double u_w = 1.0 - (q[2] - z_s), d_w = 1.0 - u_w;
    int64_t ps = sx * sy;
    double higher = t_w * (l_w * VOX(src, dt, z_s * ps + y_s * sx + x_s) + r_w * VOX(src, dt, z_s * ps + y_s * sx + x_b)) +
                    b_w * (l_w * VOX(src, dt, z_s * ps + y_b * sx + x_s) + r_w * VOX(src, dt, z_s * ps + y_b * sx + x_b));
    double lower = t_w * (l_w * VOX(src, dt, z_b * ps + y_s * sx + x_s) + r_w * VOX(src, dt, z_b * ps + y_s * sx + x_b)) +
                   b_w * (l_w * VOX(src, dt, z_b * ps + y_b * sx + x_s) + r_w * VOX(src, dt, z_b * ps + y_b * sx + x_b));
    return u_w * higher + d_w * lower;
}

static inline void store_vox(void *dst, int dt, int64_t idx, double v)
{
    /* C conversion double -> unsigned integer truncates, as the reference's
     * assignment to unsigned char does. */
    if (dt == 1) ((uint8_t *)dst)[idx] = (uint8_t)v;
    else ((uint16_t *)dst)[idx] = (uint16_t)v;
}

/* ------------------------------------------------------------------------- */
/* (a-3)+(a-4) whole-volume TPS warp from a node displacement grid            */
/* ------------------------------------------------------------------------- */

/* For every cell s < gsz-3 (chazhi.cu:632; the whole-image CPU loop runs to
 * gsz-1 at q_imgwarp_tps_quicksmallmemory.cpp:2123-2125 but every voxel of
 * the extra cells lies outside the image and is skipped):
 *   q_dfblcokinterp_bspline (:169-203): gather the 4x4x4 nodes in (z, x, y)
 *     order, multiply by the n^3 x 64 basis (double, k order), store the
 *     per-voxel DF as float in (zz, xx, yy) order;
 *   q_imgblockwarp (:85-167): pos_sub = pos_warp + DF; OOB -> 0; trilinear
 *     + 0.5 then truncation (interp 0) or nearest neighbour (interp 1).
 * src/dst are x-fastest volumes of sz0 x sz1 x sz2 (dt 1 = u8, 2 = u16).
 * df is the node grid from or_tps_grid.  threads: 1 = serial as the
 * reference's whole-image path, 0 = all cores, k = k threads. */
/* The same warp restricted to the output box [b0, b0 + bn) (global voxel
 * coordinates, inside the volume), written to dst as an x-fastest bn0 x bn1 x
 * bn2 buffer.  Only the cells that overlap the box are expanded; every
 * voxel's arithmetic is the whole-volume warp's, so a box of the whole-volume
 * output is reproduced exactly.  Used to check large volumes on a sample of
 * tiles, and to time the CPU path on a slab of planes. */
int or_tps_warp_box(const void *src, int dt, int64_t sz0, int64_t sz1, int64_t sz2,
                    const float *df, int64_t gsz0, int64_t gsz1, int64_t gsz2, int g,
                    int interp, int threads, int64_t b0x, int64_t b0y, int64_t b0z,
                    int64_t bnx, int64_t bny, int64_t bnz, void *dst)
{
    if (!src || !dst || !df || (dt != 1 && dt != 2) || g < 1) return OR_ERR_ARG;
    if (gsz0 < 4 || gsz1 < 4 || gsz2 < 4) return OR_ERR_ARG;
    if (b0x < 0 || b0y < 0 || b0z < 0 || bnx < 1 || bny < 1 || bnz < 1 || b0x + bnx > sz0 || b0y + bny > sz1 ||
        b0z + bnz > sz2)
        return OR_ERR_ARG;
    set_threads(threads);
    double *TB = (double *)malloc(sizeof(double) * 4 * (size_t)g);
    if (!TB) return OR_ERR_OOM;
    or_bspline_tb(g, TB);
    /* cells [cl, ch) that overlap the box, within s < gsz - 3 */
    const int64_t clx = b0x / g, cly = b0y / g, clz = b0z / g;
    int64_t chx = (b0x + bnx + g - 1) / g, chy = (b0y + bny + g - 1) / g, chz = (b0z + bnz + g - 1) / g;
    if (chx > gsz0 - 3) chx = gsz0 - 3;
    if (chy > gsz1 - 3) chy = gsz1 - 3;
    if (chz > gsz2 - 3) chz = gsz2 - 3;
    const int64_t ncz = chz - clz, ncy = chy - cly, ncx = chx - clx;
    const int64_t ncells = ncz > 0 && ncy > 0 && ncx > 0 ? ncz * ncy * ncx : 0;
    int rc = OR_OK;
#pragma omp parallel if (threads != 1)
    {
        float *blk = (float *)malloc(sizeof(float) * 3 * (size_t)g * g * g);
        double nodes[64][3];
        if (!blk) {
#pragma omp atomic write
            rc = OR_ERR_OOM;
        }
#pragma omp for schedule(dynamic, 4)
        for (int64_t cell = 0; cell < ncells; ++cell) {
            if (!blk) continue;
            int64_t scz = clz + cell / (ncy * ncx);
            int64_t scy = cly + (cell / ncx) % ncy;
            int64_t scx = clx + cell % ncx;
            /* gather in (dep, col, row) = (z, x, y) order */
            int ind = 0;
            for (int64_t dep = scz; dep < scz + 4; ++dep)
                for (int64_t cx = scx; cx < scx + 4; ++cx)
                    for (int64_t ry = scy; ry < scy + 4; ++ry) {
                        const float *nd = df + 3 * (size_t)((dep * gsz1 + ry) * gsz0 + cx);
                        nodes[ind][0] = nd[0];
                        nodes[ind][1] = nd[1];
                        nodes[ind][2] = nd[2];
                        ++ind;
                    }
            /* x_bsplinebasis * gridblock; row = (zz*n + xx)*n + yy,
             * col = (dz*4 + dx)*4 + dy */
            for (int zz = 0; zz < g; ++zz)
                for (int xx = 0; xx < g; ++xx)
                    for (int yy = 0; yy < g; ++yy) {
                        double a0 = 0, a1 = 0, a2 = 0;
                        int k = 0;
                        for (int dz = 0; dz < 4; ++dz)
                            for (int dx = 0; dx < 4; ++dx) {
                                double bzx = TB[zz * 4 + dz] * TB[xx * 4 + dx];
                                for (int dy = 0; dy < 4; ++dy, ++k) {
                                    double w = bzx * TB[yy * 4 + dy];
                                    a0 += w * nodes[k][0];
                                    a1 += w * nodes[k][1];
                                    a2 += w * nodes[k][2];
                                }
                            }
                        float *o = blk + 3 * (size_t)((zz * g + yy) * g + xx);
                        o[0] = (float)a0;
                        o[1] = (float)a1;
                        o[2] = (float)a2;
                    }
            /* q_imgblockwarp */
            int64_t start_x = scx * g, start_y = scy * g, start_z = scz * g;
            for (int z = 0; z < g; ++z)
                for (int y = 0; y < g; ++y)
                    for (int x = 0; x < g; ++x) {
                        int64_t pw0 = start_x + x, pw1 = start_y + y, pw2 = start_z + z;
                        if (pw0 >= sz0 || pw1 >= sz1 || pw2 >= sz2) continue;
                        if (pw0 < b0x || pw1 < b0y || pw2 < b0z || pw0 >= b0x + bnx || pw1 >= b0y + bny ||
                            pw2 >= b0z + bnz)
                            continue;
                        const float *o = blk + 3 * (size_t)((z * g + y) * g + x);
                        double q[3];
                        q[0] = pw0 + (double)o[0];
                        q[1] = pw1 + (double)o[1];
                        q[2] = pw2 + (double)o[2];
                        int64_t oi = ((pw2 - b0z) * bny + (pw1 - b0y)) * bnx + (pw0 - b0x);
                        if (q[0] < 0 || q[0] > sz0 - 1 || q[1] < 0 || q[1] > sz1 - 1 || q[2] < 0 || q[2] > sz2 - 1) {
                            store_vox(dst, dt, oi, 0.0);
                            continue;
                        }
                        if (interp == 1) {
                            int64_t nn[3];
                            int64_t szv[3] = {sz0, sz1, sz2};
                            for (int i = 0; i < 3; ++i) {
                                nn[i] = (int64_t)(q[i] + 0.5);
                                nn[i] = nn[i] < szv[i] ? nn[i] : szv[i] - 1;
                            }
                            store_vox(dst, dt, oi, VOX(src, dt, (nn[2] * sz1 + nn[1]) * sz0 + nn[0]));
                        } else {
                            store_vox(dst, dt, oi, trilinear(src, dt, sz0, sz1, q) + 0.5);
                        }
                    }
        }
        free(blk);
    }
    free(TB);
    return rc;
}

/* The whole-volume warp described above: the box is the whole volume. */
int or_tps_warp(const void *src, int dt, int64_t sz0, int64_t sz1, int64_t sz2,
                const float *df, int64_t gsz0, int64_t gsz1, int64_t gsz2, int g,
                int interp, int threads, void *dst)
{
    return or_tps_warp_box(src, dt, sz0, sz1, sz2, df, gsz0, gsz1, gsz2, g, interp, threads, 0, 0, 0, sz0, sz1,
                           sz2, dst);
}

/* ------------------------------------------------------------------------- */
/* (a-5) affine fit (3-D DLT with Hartley normalisation) and resample         */
/* ------------------------------------------------------------------------- */

/* q_normalize_points_3D (q_warp_affine_tps.cpp:493-570): centre on the
 * centroid, scale so that the mean distance to the origin is 1. */
static void normalize_points(int n, const double *p, double *out, double N[16])
{
    double cx = 0, cy = 0, cz = 0;
    for (int i = 0; i < n; ++i) { cx += p[3 * i]; cy += p[3 * i + 1]; cz += p[3 * i + 2]; }
    cx /= n; cy /= n; cz /= n;
    double avg = 0;
    for (int i = 0; i < n; ++i) {
        out[3 * i] = p[3 * i] - cx;
        out[3 * i + 1] = p[3 * i + 1] - cy;
        out[3 * i + 2] = p[3 * i + 2] - cz;
        avg += sqrt(out[3 * i] * out[3 * i] + out[3 * i + 1] * out[3 * i + 1] + out[3 * i + 2] * out[3 * i + 2]);
    }
    avg /= n;
    double s = 1.0 / avg;
    for (int i = 0; i < 3 * n; ++i) out[i] *= s;
    memset(N, 0, sizeof(double) * 16);
    N[0] = s; N[3] = -s * cx;
    N[5] = s; N[7] = -s * cy;
    N[10] = s; N[11] = -s * cz;
    N[15] = 1;
}

static int inv4(const double *m, double *inv)
{
    double a[16], b[16];
    memcpy(a, m, sizeof(a));
    for (int i = 0; i < 16; ++i) b[i] = (i % 5 == 0) ? 1.0 : 0.0;
    for (int k = 0; k < 4; ++k) {
        int p = k;
        for (int i = k + 1; i < 4; ++i)
            if (fabs(a[i * 4 + k]) > fabs(a[p * 4 + k])) p = i;
        if (a[p * 4 + k] == 0.0) return OR_ERR_SINGULAR;
        for (int j = 0; j < 4; ++j) {
            double t = a[k * 4 + j]; a[k * 4 + j] = a[p * 4 + j]; a[p * 4 + j] = t;
            t = b[k * 4 + j]; b[k * 4 + j] = b[p * 4 + j]; b[p * 4 + j] = t;
        }
        double piv = a[k * 4 + k];
        for (int j = 0; j < 4; ++j) { a[k * 4 + j] /= piv; b[k * 4 + j] /= piv; }
        for (int i = 0; i < 4; ++i) {
            if (i == k) continue;
            double f = a[i * 4 + k];
            for (int j = 0; j < 4; ++j) { a[i * 4 + j] -= f * a[k * 4 + j]; b[i * 4 + j] -= f * b[k * 4 + j]; }
        }
    }
    memcpy(inv, b, sizeof(b));
    return OR_OK;
}

static void mat4_mul(const double *a, const double *b, double *c)
{
    double t[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += a[i * 4 + k] * b[k * 4 + j];
            t[i * 4 + j] = s;
        }
    memcpy(c, t, sizeof(t));
}

/* q_affine_compute_affinmatrix_3D (q_warp_affine_tps.cpp:649-731): fit
 * B = T A from n >= 4 pairs.  Normalise both sets, build the 3n x 13 DLT
 * matrix, take the right singular vector of the smallest singular value
 * (newmat SVD), divide by h13, reshape to 4x4 and de-normalise:
 * T = NB^-1 H NA.  The SVD is computed here by one-sided Jacobi in FP64.
 * ptsA = target points, ptsB = subject points (the reference's call at
 * q_warp_affine_tps.cpp:1351), so T maps target -> subject. */
int or_affine_fit(int n, const double *ptsA, const double *ptsB, double *T)
{
    if (n < 4 || !ptsA || !ptsB || !T) return OR_ERR_ARG;
    double *An = (double *)malloc(sizeof(double) * 3 * n);
    double *Bn = (double *)malloc(sizeof(double) * 3 * n);
    int rows = 3 * n;
    double *M = (double *)calloc((size_t)rows * 13, sizeof(double));
    if (!An || !Bn || !M) { free(An); free(Bn); free(M); return OR_ERR_OOM; }
    double NA[16], NB[16];
    normalize_points(n, ptsA, An, NA);
    normalize_points(n, ptsB, Bn, NB);
    for (int i = 0; i < n; ++i) {
        double *r0 = M + (size_t)(3 * i) * 13, *r1 = r0 + 13, *r2 = r1 + 13;
        r0[0] = An[3 * i]; r0[1] = An[3 * i + 1]; r0[2] = An[3 * i + 2]; r0[3] = 1.0; r0[12] = -Bn[3 * i];
        r1[4] = An[3 * i]; r1[5] = An[3 * i + 1]; r1[6] = An[3 * i + 2]; r1[7] = 1.0; r1[12] = -Bn[3 * i + 1];
        r2[8] = An[3 * i]; r2[9] = An[3 * i + 1]; r2[10] = An[3 * i + 2]; r2[11] = 1.0; r2[12] = -Bn[3 * i + 2];
    }
    /* one-sided Jacobi on the columns of M: M V = U S */
    double V[13 * 13];
    for (int i = 0; i < 169; ++i) V[i] = (i % 14 == 0) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < 12; ++p)
            for (int q = p + 1; q < 13; ++q) {
                double a = 0, b = 0, c = 0;
                for (int r = 0; r < rows; ++r) {
                    double mp = M[(size_t)r * 13 + p], mq = M[(size_t)r * 13 + q];
                    a += mp * mp; b += mq * mq; c += mp * mq;
                }
                if (fabs(c) <= 1e-300) continue;
                double rel = fabs(c) / sqrt(a * b);
                if (rel > off) off = rel;
                if (rel < 1e-15) continue;
                double zeta = (b - a) / (2.0 * c);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
                for (int r = 0; r < rows; ++r) {
                    double mp = M[(size_t)r * 13 + p], mq = M[(size_t)r * 13 + q];
                    M[(size_t)r * 13 + p] = cs * mp - sn * mq;
                    M[(size_t)r * 13 + q] = sn * mp + cs * mq;
                }
                for (int r = 0; r < 13; ++r) {
                    double vp = V[r * 13 + p], vq = V[r * 13 + q];
                    V[r * 13 + p] = cs * vp - sn * vq;
                    V[r * 13 + q] = sn * vp + cs * vq;
                }
            }
        if (off < 1e-15) break;
    }
    int best = 0;
    double bestn = -1;
    for (int p = 0; p < 13; ++p) {
        double s = 0;
        for (int r = 0; r < rows; ++r) s += M[(size_t)r * 13 + p] * M[(size_t)r * 13 + p];
        if (bestn < 0 || s < bestn) { bestn = s; best = p; }
    }
    double h[13];
    for (int i = 0; i < 13; ++i) h[i] = V[i * 13 + best];
    int rc = OR_OK;
    if (h[12] == 0.0) rc = OR_ERR_SINGULAR;
    else {
        for (int i = 0; i < 13; ++i) h[i] /= h[12];
        double H[16] = {h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7], h[8], h[9], h[10], h[11], 0, 0, 0, 1};
        double NBi[16];
        rc = inv4(NB, NBi);
        if (!rc) {
            double tmp[16];
            mat4_mul(NBi, H, tmp);
            mat4_mul(tmp, NA, T);
        }
    }
    free(An); free(Bn); free(M);
    return rc;
}

/* Whole-image affine resample (q_warp_affine_tps.cpp:1373-1437): for every
 * output voxel (x,y,z) of the output box, q = M [x y z 1]'; OOB -> 0;
 * trilinear; truncation (no +0.5).  interp 1 = nearest neighbour with the
 * TPS path's rule (+0.5, clamp).  Output dims may differ from the source
 * (resize / downsample).  threads 0 = all cores (the reference's OpenMP
 * over x at :1375). */
int or_affine_warp(const void *src, int dt, int64_t sz0, int64_t sz1, int64_t sz2,
                   const double *Mx, int interp, int threads,
                   void *dst, int64_t dz0, int64_t dz1, int64_t dz2)
{
    if (!src || !dst || !Mx || (dt != 1 && dt != 2)) return OR_ERR_ARG;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) if (threads != 1)
    for (int64_t z = 0; z < dz2; ++z)
        for (int64_t y = 0; y < dz1; ++y)
            for (int64_t x = 0; x < dz0; ++x) {
                double q[3];
                for (int r = 0; r < 3; ++r)
                    q[r] = Mx[r * 4 + 0] * x + Mx[r * 4 + 1] * y + Mx[r * 4 + 2] * z + Mx[r * 4 + 3] * 1.0;
                int64_t oi = (z * dz1 + y) * dz0 + x;
                if (q[0] < 0 || q[0] > sz0 - 1 || q[1] < 0 || q[1] > sz1 - 1 || q[2] < 0 || q[2] > sz2 - 1) {
                    store_vox(dst, dt, oi, 0.0);
                    continue;
                }
                if (interp == 1) {
                    int64_t nn[3];
                    int64_t szv[3] = {sz0, sz1, sz2};
                    for (int i = 0; i < 3; ++i) {
                        nn[i] = (int64_t)(q[i] + 0.5);
                        nn[i] = nn[i] < szv[i] ? nn[i] : szv[i] - 1;
                    }
                    store_vox(dst, dt, oi, VOX(src, dt, (nn[2] * sz1 + nn[1]) * sz0 + nn[0]));
                } else {
                    store_vox(dst, dt, oi, trilinear(src, dt, sz0, sz1, q));
                }
            }
    return OR_OK;
}

/* Downsample factor of q_imagewarp_affine_cyf_downsample
 * (q_warp_affine_tps.cpp:1477-1479): maxdim/600 rounded half up. */
int or_downsample_factor(int64_t sz0, int64_t sz1, int64_t sz2)
{
    int64_t f = sz0 > sz1 ? (sz0 > sz2 ? sz0 : sz2) : (sz1 > sz2 ? sz1 : sz2);
    return (int)(f / 600 + (f % 600 >= 300 ? 1 : 0));
}
