// tw_solve.cu -- FP64 landmark solves on sm_100a: the regularised TPS system
// and the 3-D affine DLT fit.
//
// TPS (reference: compute_df_stps_subsampled_volume_4bspline,
// q_imgwarp_tps_quicksmallmemory.cpp:377-588, whose GPU branch runs cuSOLVER
// Sgeqrf on an N x N zero-padded copy of X (qr.cu:8-130), N-4 host round trips
// of Gram-Schmidt (extendornormal.cu:55-150), four cublasSgemm calls with a
// handle created per call (aff.cu:37-133) and an unpivoted FP32 Gauss-Jordan
// inverse with 3(N-4) launches (GET_A_i.cu:80-161), all in FP32):
//
//   c = q2 (q2' K q2 + lambda I)^-1 q2' Y,   d = r^-1 q1' (Y - K c)
//
// is computed here entirely in FP64 without ever forming K, Q or A^-1:
//   1. Householder QR of X = [1 s] (n x 4): 4 reflectors H_k = I - tau v v'.
//      Q = H1 H2 H3 H4; q1 = Q(:,0:4), q2 = Q(:,4:n).  c and d do not depend
//      on which orthonormal basis q2 is (the reference completes q1 by
//      Gram-Schmidt instead), only on span(q2) = span(X)^perp.
//   2. Q' K Q by four symmetric rank-2 updates: H K H = K - v w' - w v' with
//      w = tau p - (tau^2 v'p / 2) v, p = K v.  All four p come from one
//      product P0 = K V over the implicit K_ij = -|s_i - s_j|.
//   3. A = (Q' K Q)(4:,4:) + lambda I is symmetric positive definite (-|r| is
//      conditionally positive definite of order 1 in 3-D and q2 is orthogonal
//      to the polynomials), so it is factored by a blocked right-looking
//      Cholesky: diagonal block in shared memory, panel TRSM, trailing SYRK
//      in 64 x 64 FP64 tiles.
//   4. z = Q' Y; w = A^-1 z(4:): the forward substitution rides along in the
//      factorisation (z(4:)' is an extra row block of the panel solves and
//      trailing updates), the back substitution is one CTA;
//      c = Q [0; w]; d = R^-1 (Q' (Y - K c))(0:4).
//
// Affine (reference: q_affine_compute_affinmatrix_3D,
// q_warp_affine_tps.cpp:649-731, newmat SVD of the 3N x 13 DLT matrix):
// one CTA normalises both point sets, accumulates the 13 x 13 normal matrix
// in FP64 and takes the eigenvector of its smallest eigenvalue by cyclic
// Jacobi, which is the right singular vector the reference uses.

#include "tw_internal.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace tw {

namespace {

constexpr int kNB = 64;          // Cholesky block
constexpr int kRedThreads = 1024;

// status word bits
constexpr int kStSingularX = 1;
constexpr int kStNotSPD = 2;

__device__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < nw; ++i) t += sh[i];
    return t;
}

__device__ __forceinline__ double kdist(const double *ctr, int i, int j)
{
    double dx = ctr[3 * i] - ctr[3 * j];
    double dy = ctr[3 * i + 1] - ctr[3 * j + 1];
    double dz = ctr[3 * i + 2] - ctr[3 * j + 2];
    return -sqrt(dx * dx + dy * dy + dz * dz);
}

// 1. Householder QR of X = [1 s].  Xw (n x 4) is a work copy; V (n x 4) gets
// the reflectors (zeros above the diagonal), tau[4], R[16].
__global__ void k_qr(const double *ctr, int n, double *Xw, double *V, double *tau, double *R, int *status)
{
    __shared__ double sh[32];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        Xw[i * 4 + 0] = 1.0;
        Xw[i * 4 + 1] = ctr[3 * i];
        Xw[i * 4 + 2] = ctr[3 * i + 1];
        Xw[i * 4 + 3] = ctr[3 * i + 2];
    }
    __syncthreads();
    double colnorm[4];
    for (int j = 0; j < 4; ++j) {
        double s = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) s += Xw[i * 4 + j] * Xw[i * 4 + j];
        colnorm[j] = sqrt(block_sum(s, sh));
    }
    for (int k = 0; k < 4; ++k) {
        double s = 0.0;
        for (int i = k + threadIdx.x; i < n; i += blockDim.x) s += Xw[i * 4 + k] * Xw[i * 4 + k];
        const double nrm2 = block_sum(s, sh);
        const double nrm = sqrt(nrm2);
        const double xkk = Xw[k * 4 + k];
        const double alpha = xkk > 0 ? -nrm : nrm;
        const double vk = xkk - alpha;
        const double vv = nrm2 - xkk * xkk + vk * vk;
        const double t = vv > 0 ? 2.0 / vv : 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            V[i * 4 + k] = i < k ? 0.0 : (i == k ? vk : Xw[i * 4 + k]);
        __syncthreads();
        if (threadIdx.x == 0) {
            tau[k] = t;
            R[k * 4 + k] = alpha;
            for (int j = 0; j < k; ++j) R[k * 4 + j] = 0.0;
            if (!(fabs(alpha) > 1e-10 * (colnorm[k] + 1e-300))) atomicOr(status, kStSingularX);
        }
        for (int j = k; j < 4; ++j) {
            double d = 0.0;
            for (int i = k + threadIdx.x; i < n; i += blockDim.x) d += V[i * 4 + k] * Xw[i * 4 + j];
            const double sj = t * block_sum(d, sh);
            for (int i = k + threadIdx.x; i < n; i += blockDim.x) Xw[i * 4 + j] -= sj * V[i * 4 + k];
            __syncthreads();
            if (threadIdx.x == 0 && j > k) R[k * 4 + j] = Xw[k * 4 + j];
        }
        __syncthreads();
    }
}

// out (n x 4) = K B for the implicit K_ij = -|s_i - s_j|; one warp per row.
__global__ void k_kmul(const double *ctr, int n, const double *B, double *out)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (int j = lane; j < n; j += 32) {
        const double k = kdist(ctr, warp, j);
        a0 += k * B[j * 4 + 0];
        a1 += k * B[j * 4 + 1];
        a2 += k * B[j * 4 + 2];
        a3 += k * B[j * 4 + 3];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        a3 += __shfl_xor_sync(0xffffffffu, a3, o);
    }
    if (lane == 0) {
        out[warp * 4 + 0] = a0;
        out[warp * 4 + 1] = a1;
        out[warp * 4 + 2] = a2;
        out[warp * 4 + 3] = a3;
    }
}

// 2. From P0 = K V derive the rank-2 update vectors W (n x 4), and Z = Q' Y.
__global__ void k_wvec(int n, const double *V, const double *tau, const double *P0, double *W, const double *Y,
                       double *Z)
{
    __shared__ double sh[32];
    __shared__ double wv[4][4], vvd[4][4];  // w_j . v_k, v_j . v_k
    for (int k = 0; k < 4; ++k) {
        // p_k = P0_k - sum_{j<k} [ v_j (w_j . v_k) + w_j (v_j . v_k) ]
        for (int j = 0; j < k; ++j) {
            double a = 0, b = 0;
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                a += W[i * 4 + j] * V[i * 4 + k];
                b += V[i * 4 + j] * V[i * 4 + k];
            }
            a = block_sum(a, sh);
            b = block_sum(b, sh);
            if (threadIdx.x == 0) { wv[j][k] = a; vvd[j][k] = b; }
        }
        __syncthreads();
        double beta = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double p = P0[i * 4 + k];
            for (int j = 0; j < k; ++j) p -= V[i * 4 + j] * wv[j][k] + W[i * 4 + j] * vvd[j][k];
            W[i * 4 + k] = p;  // temporarily p
            beta += V[i * 4 + k] * p;
        }
        beta = block_sum(beta, sh);
        const double t = tau[k];
        const double cf = 0.5 * t * t * beta;
        for (int i = threadIdx.x; i < n; i += blockDim.x) W[i * 4 + k] = t * W[i * 4 + k] - cf * V[i * 4 + k];
        __syncthreads();
    }
    // Z = H4 H3 H2 H1 Y
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int c = 0; c < 4; ++c) Z[i * 4 + c] = Y[i * 4 + c];
    __syncthreads();
    for (int k = 0; k < 4; ++k) {
        for (int c = 0; c < 4; ++c) {
            double d = 0.0;
            for (int i = threadIdx.x; i < n; i += blockDim.x) d += V[i * 4 + k] * Z[i * 4 + c];
            d = tau[k] * block_sum(d, sh);
            for (int i = threadIdx.x; i < n; i += blockDim.x) Z[i * 4 + c] -= d * V[i * 4 + k];
            __syncthreads();
        }
    }
}

// The factorisation works on an (m + 4) x m row-major array: rows 0..m-1
// hold A, rows m..m+3 hold the four right-hand sides z(4:) transposed.  Row
// block ib < nblk covers rows 64 ib.., the extra row block nblk covers the
// four right-hand-side rows.  The right-looking Cholesky treats that block like
// any other row below the diagonal, so its panel solves and trailing updates
// perform the forward substitution y = L^-1 z(4:) as part of the
// factorisation, in parallel with it; rows m..m+3 end up holding y'.
__device__ __forceinline__ int row_block_start(int ib, int nblk, int m) { return ib < nblk ? ib * kNB : m; }
__device__ __forceinline__ int row_block_rows(int ib, int nblk, int m)
{
    return ib < nblk ? min(kNB, m - ib * kNB) : 4;
}

// 3a. A = (Q'KQ)(4:,4:) + lambda I, and the right-hand-side rows z(4:)'
__global__ void k_fill_a(const double *__restrict__ ctr, int n, const double *__restrict__ V,
                         const double *__restrict__ W, const double *__restrict__ Z, double lambda,
                         double *__restrict__ A)
{
    const int m = n - 4;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= m + 4 || j >= m) return;
    if (i >= m) {
        A[(size_t)i * m + j] = Z[(j + 4) * 4 + (i - m)];
        return;
    }
    const int gi = i + 4, gj = j + 4;
    double v = kdist(ctr, gi, gj);
#pragma unroll
    for (int k = 0; k < 4; ++k) v -= V[gi * 4 + k] * W[gj * 4 + k] + W[gi * 4 + k] * V[gj * 4 + k];
    if (i == j) v += lambda;
    A[(size_t)i * m + j] = v;
}

// ---- 3b-4b: one cooperative kernel, one CTA of 256 threads per SM.
//
// The tiled right-looking Cholesky and both substitutions run as tasks on
// 64 x 64 tiles, ordered by dependency counters in global memory instead of
// grid-wide barriers: POTRF(k) factors diagonal tile k once every update of
// it has landed; TRSM(i, k) solves row block i of panel k (the right-hand-side
// block included) once POTRF(k) and the updates of tile (i, k) are done;
// UPDATE(i, j, k) subtracts L(i,k) L(j,k)' from tile (i, j) once both panel
// tiles exist and the tile's previous update is in.  The back substitution
// is DIAG(kb) (the diagonal block's triangular solve) and BACK(ib, kb) (the
// rows of block ib) in the same way.
//
// The critical path is the chain POTRF(k-1) -> TRSM(k, k-1) -> UPDATE(k, k,
// k-1) -> POTRF(k): CTA 0 runs only that chain, one fused step per k with
// its three tiles kept in shared memory, and then the back substitution's
// chain.  The other CTAs take every other task in one order that respects
// every dependency, CTA c taking every (G-1)-th; as all CTAs are resident
// (cooperative launch) and every wait of a task is on tasks earlier in that
// order, the lowest unfinished task can always run, so the schedule cannot
// deadlock.  L1 is not coherent across SMs within a kernel, so every load of
// data another CTA wrote (A, z) bypasses L1 (__ldcg).

constexpr int kSolveThreads = 256;
constexpr int kStTimeout = 4;
// A CTA gives up on a dependency after limit_ns (the context's
// solve_barrier_ns, 30 s unless a test shortened it).  The launch is
// cooperative, so every CTA can be resident at once; while other work (the
// previous job's resample, a caller's kernel on another stream) still holds
// SMs, some CTAs start later than others and the early ones wait, so the
// bound is generous, but it is a bound.

// Dependency counters (zeroed before the launch); tdone[nblk + 1] (panel
// tiles solved per row block), cnt[(nblk + 1) nblk] (updates applied per
// tile) and bcnt[nblk] (back-substitution updates applied per row block)
// follow in the same allocation.
struct SolveFlags {
    int err;    // set by a CTA that gave up waiting
    int pdone;  // diagonal tiles factored
    int ddone;  // back-substitution diagonal blocks solved, from the last block down
    int pad;
};

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0 waits until *flag >= want; every thread returns true, or false
// (on every thread) when this or another CTA gave up.
__device__ bool wait_ge(const int *flag, int want, SolveFlags *F, int *status, unsigned long long limit_ns)
{
    __shared__ int ok_sh;
    if (threadIdx.x == 0) {
        int ok = 1;
        if (ld_acquire(flag) < want) {
            const unsigned long long t0 = globaltimer_ns();
            while (ld_acquire(flag) < want) {
                if (*reinterpret_cast<volatile int *>(&F->err) || globaltimer_ns() - t0 > limit_ns) {
                    atomicOr(&F->err, 1);
                    atomicOr(status, kStTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        ok_sh = ok;
    }
    __syncthreads();
    return ok_sh != 0;
}

// Publishes a finished task: every thread's writes, then *flag = value.
__device__ __forceinline__ void signal_done(int *flag, int value)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release(flag, value);
    }
}

// Column J onwards of the Cholesky of a 16 x 16 block held by the lanes of
// one warp, lane l (l = lane % 16) owning row l (v[k] = element (l, k)): the
// pivot comes from its row's lane, the scaled column goes to the other lanes
// by shuffles.  Compile-time recursion over the columns keeps every index of
// v constant, so v stays in registers.
template <int J>
__device__ __forceinline__ void panel_factor(double (&v)[16], int l, int lane, int *status)
{
    if constexpr (J < 16) {
        const unsigned full = 0xffffffffu;
        double d = __shfl_sync(full, v[J], J);  // the pivot, from its row's lane
        if (!(d > 0.0)) {
            if (lane == 0) atomicOr(status, kStNotSPD);
            d = 1.0;
        }
        const double inv = rsqrt(d);
        if (l > J) v[J] *= inv;
        else if (l == J) v[J] = d * inv;
#pragma unroll
        for (int k = J + 1; k < 16; ++k) {
            const double lkj = __shfl_sync(full, v[J], k);  // L(k, J), from row k's lane
            if (l >= k) v[k] -= v[J] * lkj;
        }
        panel_factor<J + 1>(v, l, lane, status);
    }
}

// Cholesky of a diagonal tile held in shared memory (lower triangle of
// a[kNB][kNB + 1]; padding rows and columns hold the identity), in four
// 16-column panels: warp 0 factors the panel's 16 x 16 diagonal block in
// registers (lane l < 16 owns its row l; each finished column goes to the
// other lanes by shuffles), then every thread solves the panel's rows below
// it (four lanes per row) and applies the trailing update.  rdiag gets the
// reciprocals of the diagonal.  Three CTA barriers per panel.
__device__ void potrf_smem(double (*a)[kNB + 1], double *rdiag, int *status)
{
    const int t = threadIdx.x, lane = t & 31;
    const unsigned full = 0xffffffffu;
#pragma unroll 1
    for (int c0 = 0; c0 < kNB; c0 += 16) {
        if (t < 32) {
            const int l = lane & 15;
            double v[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] = k <= l ? a[c0 + l][c0 + k] : 0.0;
            panel_factor<0>(v, l, lane, status);
            if (lane < 16) {
                double dl = 1.0;  // v[l], selected without a run-time index (v stays in registers)
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    if (k <= l) a[c0 + l][c0 + k] = v[k];
                    if (k == l) dl = v[k];
                }
                rdiag[c0 + l] = 1.0 / dl;
            }
        }
        __syncthreads();
        const int nr = kNB - c0 - 16;  // rows below the panel's diagonal block
        {
            // X(i, c0 + c) = (A(i, c0 + c) - sum_{k<c} X(i, c0 + k) L(c0 + c, c0 + k)) / L(c0 + c, c0 + c)
            const int r = t >> 2, q = t & 3, base = lane & ~3;
            const bool act = r < nr;
            const int i = c0 + 16 + (act ? r : 0);
            double x[4];
#pragma unroll
            for (int k4 = 0; k4 < 4; ++k4) x[k4] = act ? a[i][c0 + 4 * k4 + q] : 0.0;
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const double mine = x[c >> 2] * rdiag[c0 + c];  // meaningful in the owner lane only
                const double xc = __shfl_sync(full, mine, base | (c & 3));
                if (act && q == (c & 3)) a[i][c0 + c] = xc;
#pragma unroll
                for (int k4 = 0; k4 < 4; ++k4) {
                    const int cp = 4 * k4 + q;
                    if (cp > c) x[k4] -= xc * a[c0 + cp][c0 + c];
                }
            }
        }
        __syncthreads();
        for (int e = t; e < nr * nr; e += blockDim.x) {
            const int ii = e / nr, jj = e % nr;
            if (jj <= ii) {
                const int i = c0 + 16 + ii, j = c0 + 16 + jj;
                double acc = 0.0;
#pragma unroll
                for (int k = 0; k < 16; ++k) acc += a[i][c0 + k] * a[j][c0 + k];
                a[i][j] -= acc;
            }
        }
        __syncthreads();
    }
}

// Loads tile (row block ib, column block jb) of A into t (rows x cols of it
// valid; the rest: identity on the diagonal when `diag`, else zero).
__device__ void load_tile(double (*t)[kNB + 1], const double *__restrict__ A, int m, int i0, int rows, int j0, int cols,
                          bool diag)
{
#pragma unroll 4
    for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
        const int r = e / kNB, c = e % kNB;
        t[r][c] = (r < rows && c < cols) ? __ldcg(&A[(size_t)(i0 + r) * m + j0 + c])
                                         : ((diag && r == c) ? 1.0 : 0.0);
    }
}

__device__ void store_tile(double *__restrict__ A, int m, const double (*t)[kNB + 1], int i0, int rows, int j0, int cols,
                           bool lower)
{
    for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
        const int r = e / kNB, c = e % kNB;
        if (r < rows && c < cols) A[(size_t)(i0 + r) * m + j0 + c] = (!lower || c <= r) ? t[r][c] : 0.0;
    }
}

// X = X L^-T for a tile X in shared memory against a factored diagonal tile
// L (rdiag: reciprocals of its diagonal), nbk valid columns.  Rows are
// independent: the four lanes (q = lane & 3) of one row keep its columns q,
// q+4, .. in registers; column c is finished by its owner (x 1/L(c,c)),
// handed to the other three by a warp shuffle, and subtracted from the later
// columns: X(r,c') -= X(r,c) L(c',c).  No CTA barrier inside the column loop.
__device__ void trsm_smem(const double (*L)[kNB + 1], double (*X)[kNB + 1], const double *rdiag, int nbk)
{
    const int lane = threadIdx.x & 31;
    const int r = (threadIdx.x >> 5) * 8 + (lane >> 2);  // 8 rows per warp
    const int q = lane & 3;
    const int base = lane & ~3;
    double x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = X[r][4 * k + q];
    // fully unrolled so that every index into x is a constant (x stays in
    // registers); columns at or beyond nbk are skipped
#pragma unroll
    for (int c = 0; c < kNB; ++c) {
        if (c >= nbk) break;
        const double mine = x[c >> 2] * rdiag[c];  // meaningful in the owner lane only
        const double xc = __shfl_sync(0xffffffffu, mine, base | (c & 3));
        if (q == (c & 3)) X[r][c] = xc;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int cp = 4 * k + q;
            if (cp > c && cp < nbk) x[k] -= xc * L[cp][c];
        }
    }
}

// acc[u][v] = sum_p Li(tr + 16u, p) Lj(tc + 16v, p) over nbk columns, thread
// (tr, tc) = (t / 16, t % 16): conflict-free reads of Lj with the 65-double pitch.
__device__ __forceinline__ void syrk_acc(const double (*Li)[kNB + 1], const double (*Lj)[kNB + 1], int nbk,
                                         double (&acc)[4][4])
{
    const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
    for (int p = 0; p < nbk; ++p) {
        double a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a[u] = Li[tr + 16 * u][p];
            b[u] = Lj[tc + 16 * u][p];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
    }
}

// trsm of row block ib against diagonal block kb: L(ib,kb) = A(ib,kb) L(kb,kb)^-T.
__device__ void trsm_tile(double *__restrict__ A, int m, int kb, int ib, double *sm)
{
    double(*L)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm);
    double(*X)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm + kNB * (kNB + 1));
    double *rdiag = sm + 2 * kNB * (kNB + 1);
    const int nblk = (m + kNB - 1) / kNB;
    const int r0 = kb * kNB;
    const int i0 = row_block_start(ib, nblk, m);
    const int nbk = min(kNB, m - r0);
    const int nbi = row_block_rows(ib, nblk, m);
    __syncthreads();
    load_tile(L, A, m, r0, nbk, r0, nbk, true);
    load_tile(X, A, m, i0, nbi, r0, nbk, false);
    __syncthreads();
    if (threadIdx.x < kNB) rdiag[threadIdx.x] = 1.0 / L[threadIdx.x][threadIdx.x];
    __syncthreads();
    trsm_smem(L, X, rdiag, nbk);
    __syncthreads();
    store_tile(A, m, X, i0, nbi, r0, nbk, false);
}

// Trailing update of tile (ib, jb) at step kb: A(ib,jb) -= L(ib,kb) L(jb,kb)' for
// kb < jb <= ib, jb a column block and ib a row block (the right-hand-side
// block included); each thread owns a 4 x 4 patch.
__device__ void syrk_tile(double *__restrict__ A, int m, int kb, int ib, int jb, double *sm)
{
    double(*Li)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm);
    double(*Lj)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm + kNB * (kNB + 1));
    const int nblk = (m + kNB - 1) / kNB;
    const int r0 = kb * kNB, i0 = row_block_start(ib, nblk, m), j0 = jb * kNB;
    const int nbk = min(kNB, m - r0), nbi = row_block_rows(ib, nblk, m), nbj = min(kNB, m - j0);
    __syncthreads();
    load_tile(Li, A, m, i0, nbi, r0, nbk, false);
    load_tile(Lj, A, m, j0, nbj, r0, nbk, false);
    __syncthreads();
    double acc[4][4];
    syrk_acc(Li, Lj, nbk, acc);
    const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            int r = tr + 16 * u, c = tc + 16 * v;
            if (r < nbi && c < nbj && (ib != jb || c <= r)) {
                double *dst = &A[(size_t)(i0 + r) * m + j0 + c];
                *dst = __ldcg(dst) - acc[u][v];
            }
        }
}

// Back substitution, diagonal block kb (CTA 0): solve D' x = z(block) for the
// four right-hand sides; warp c takes right-hand side c, lane l rows l and
// l + 32; row j of D is column j of D'.  x overwrites z(block).
__device__ void bwd_diag(const double *__restrict__ A, int m, int kb, double *__restrict__ z, double *sm)
{
    double(*D)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm);
    double *dinv = sm + kNB * (kNB + 1);
    const int r0 = kb * kNB, nb = min(kNB, m - r0);
    __syncthreads();
#pragma unroll 4
    for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
        const int r = e / kNB, c = e % kNB;
        D[r][c] = (r < nb && c <= r) ? __ldcg(&A[(size_t)(r0 + r) * m + r0 + c]) : 0.0;
    }
    if (threadIdx.x < nb) dinv[threadIdx.x] = 1.0 / __ldcg(&A[(size_t)(r0 + threadIdx.x) * m + r0 + threadIdx.x]);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < 4) {
        double b0 = lane < nb ? __ldcg(&z[(r0 + lane) * 4 + warp]) : 0.0;
        double b1 = lane + 32 < nb ? __ldcg(&z[(r0 + lane + 32) * 4 + warp]) : 0.0;
        for (int j = nb - 1; j >= 0; --j) {
            const double bj = __shfl_sync(0xffffffffu, j < 32 ? b0 : b1, j & 31);
            const double xj = bj * dinv[j];
            if (lane == (j & 31)) {
                if (j < 32) b0 = xj;
                else b1 = xj;
            }
            if (lane < j) b0 -= D[j][lane] * xj;
            if (lane + 32 < j) b1 -= D[j][lane + 32] * xj;
        }
        if (lane < nb) z[(r0 + lane) * 4 + warp] = b0;
        if (lane + 32 < nb) z[(r0 + lane + 32) * 4 + warp] = b1;
    }
}

// Back substitution, rows of block ib: z(ib) -= L(kb, ib)' x(kb), x(kb)
// already in z(kb); thread (row, rhs) accumulates over the 64 rows of L(kb, .)
// in order.
__device__ void bwd_update(const double *__restrict__ A, int m, int kb, int ib, double *__restrict__ z, double *sm)
{
    const int r0 = kb * kNB, nb = min(kNB, m - r0);
    const int i0 = ib * kNB, nbi = min(kNB, m - i0);
    double *x = sm;  // x(kb), 64 x 4
    __syncthreads();
    for (int e = threadIdx.x; e < 4 * nb; e += blockDim.x) x[e] = __ldcg(&z[r0 * 4 + e]);
    __syncthreads();
    const int il = threadIdx.x >> 2, r = threadIdx.x & 3;
    if (il < nbi) {
        double s = 0.0;
#pragma unroll 16
        for (int p = 0; p < nb; ++p) s += __ldcg(&A[(size_t)(r0 + p) * m + i0 + il]) * x[p * 4 + r];
        double *zi = &z[(i0 + il) * 4 + r];
        *zi = __ldcg(zi) - s;
    }
}

// CTA 0: the critical chain.  Step k fuses TRSM(k, k-1), UPDATE(k, k, k-1)
// and POTRF(k), keeping the factored diagonal tile, the new panel tile and
// the next diagonal tile in shared memory; then the back substitution's
// chain DIAG(kb), BACK(kb - 1, kb).
__device__ void solve_chain(double *__restrict__ A, int m, double *__restrict__ z, int *status, SolveFlags *F,
                            int *tdone, int *cnt, int *bcnt, unsigned long long limit_ns, double *sm)
{
    const int nblk = (m + kNB - 1) / kNB;
    double(*Ld)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm);
    double(*X)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm + kNB * (kNB + 1));
    double(*Ad)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(sm + 2 * kNB * (kNB + 1));
    double *rdiag = sm + 3 * kNB * (kNB + 1);
    {
        const int nb = min(kNB, m);
        load_tile(Ld, A, m, 0, nb, 0, nb, true);
        __syncthreads();
        potrf_smem(Ld, rdiag, status);
        store_tile(A, m, Ld, 0, nb, 0, nb, true);
        signal_done(&F->pdone, 1);
    }
    for (int k = 1; k < nblk; ++k) {
        const int r0 = (k - 1) * kNB, i0 = k * kNB, nbi = min(kNB, m - i0);
        // TRSM(k, k-1): X = A(k, k-1) L(k-1, k-1)^-T
        if (!wait_ge(&cnt[k * nblk + k - 1], k - 1, F, status, limit_ns)) return;
        load_tile(X, A, m, i0, nbi, r0, kNB, false);
        __syncthreads();
        trsm_smem(Ld, X, rdiag, kNB);
        __syncthreads();
        store_tile(A, m, X, i0, nbi, r0, kNB, false);
        signal_done(&tdone[k], k);
        // UPDATE(k, k, k-1): A(k, k) -= X X'
        if (!wait_ge(&cnt[k * nblk + k], k - 1, F, status, limit_ns)) return;
        load_tile(Ad, A, m, i0, nbi, i0, nbi, true);
        __syncthreads();
        {
            double acc[4][4];
            syrk_acc(X, X, kNB, acc);
            const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int r = tr + 16 * u, c = tc + 16 * v;
                    if (r < nbi && c <= r) Ad[r][c] -= acc[u][v];
                }
        }
        __syncthreads();
        // POTRF(k)
        potrf_smem(Ad, rdiag, status);
        store_tile(A, m, Ad, i0, nbi, i0, nbi, true);
        signal_done(&F->pdone, k + 1);
        double(*t)[kNB + 1] = Ld;
        Ld = Ad;
        Ad = t;
    }
    for (int kb = nblk - 1; kb >= 0; --kb) {
        if (!wait_ge(&tdone[nblk], kb + 1, F, status, limit_ns) ||
            !wait_ge(&bcnt[kb], nblk - 1 - kb, F, status, limit_ns))
            return;
        bwd_diag(A, m, kb, z, sm);
        signal_done(&F->ddone, nblk - kb);
        if (kb >= 1) {
            if (!wait_ge(&bcnt[kb - 1], nblk - 1 - kb, F, status, limit_ns)) return;
            bwd_update(A, m, kb, kb - 1, z, sm);
            signal_done(&bcnt[kb - 1], nblk - kb);
        }
    }
}

// CTAs 1 .. G-1: every other task, in one order that respects every
// dependency, CTA c taking every (G-1)-th.  Step k: the panel tiles TRSM(i, k)
// of rows i >= k + 2 (and the right-hand-side block), then the updates
// UPDATE(i, j, k) column by column, without the chain's UPDATE(k+1, k+1, k).
// Then the back substitution's BACK(ib, kb) for ib <= kb - 2.
__device__ void solve_others(double *__restrict__ A, int m, double *__restrict__ z, int *status, SolveFlags *F,
                             int *tdone, int *cnt, int *bcnt, unsigned long long limit_ns, double *sm)
{
    const int nblk = (m + kNB - 1) / kNB;
    const long long G = gridDim.x - 1, bid = blockIdx.x - 1;
    long long base = 0;  // number of the step's first task
    for (int k = 0; k < nblk; ++k) {
        const int lo_i = k + 1 < nblk ? k + 2 : k + 1;
        const int nt = nblk - lo_i + 1;
        const int first = k + 1 < nblk ? nblk - k - 1 : 0;  // updates of column block k+1, rows k+2 .. nblk
        long long nu = first;
        for (int j = k + 2; j < nblk; ++j) nu += nblk + 1 - j;
        const long long count = nt + nu;
        for (long long e = ((bid - base) % G + G) % G; e < count; e += G) {
            if (e < nt) {
                const int i = lo_i + (int)e;
                if (!wait_ge(&F->pdone, k + 1, F, status, limit_ns) ||
                    !wait_ge(&cnt[i * nblk + k], k, F, status, limit_ns))
                    return;
                trsm_tile(A, m, k, i, sm);
                if (i == nblk) {
                    // y' of block k is final: seed z(k) for the back substitution
                    __syncthreads();
                    const int r0 = k * kNB, nb = min(kNB, m - r0);
                    for (int q = threadIdx.x; q < 4 * nb; q += blockDim.x)
                        z[(r0 + (q >> 2)) * 4 + (q & 3)] = __ldcg(&A[(size_t)(m + (q & 3)) * m + r0 + (q >> 2)]);
                }
                signal_done(&tdone[i], k + 1);
            } else {
                long long f = e - nt;
                int i, j;
                if (f < first) {
                    j = k + 1;
                    i = k + 2 + (int)f;
                } else {
                    f -= first;
                    j = k + 2;
                    while (f >= nblk + 1 - j) {
                        f -= nblk + 1 - j;
                        ++j;
                    }
                    i = j + (int)f;
                }
                if (!wait_ge(&tdone[i], k + 1, F, status, limit_ns) ||
                    !wait_ge(&tdone[j], k + 1, F, status, limit_ns) ||
                    !wait_ge(&cnt[i * nblk + j], k, F, status, limit_ns))
                    return;
                syrk_tile(A, m, k, i, j, sm);
                signal_done(&cnt[i * nblk + j], k + 1);
            }
        }
        base += count;
    }
    for (int kb = nblk - 1; kb >= 0; --kb) {
        const long long count = kb >= 2 ? kb - 1 : 0;  // BACK(ib, kb) for ib = kb-2 .. 0
        for (long long e = ((bid - base) % G + G) % G; e < count; e += G) {
            const int ib = kb - 2 - (int)e;
            if (!wait_ge(&F->ddone, nblk - kb, F, status, limit_ns) ||
                !wait_ge(&bcnt[ib], nblk - 1 - kb, F, status, limit_ns))
                return;
            bwd_update(A, m, kb, ib, z, sm);
            signal_done(&bcnt[ib], nblk - kb);
        }
        base += count;
    }
}

__global__ void __launch_bounds__(kSolveThreads) k_chol_solve(double *__restrict__ A, int m, double *__restrict__ Z,
                                                              int *status, int *flags, unsigned long long limit_ns)
{
    extern __shared__ double sm[];
    const int nblk = (m + kNB - 1) / kNB;
    SolveFlags *F = reinterpret_cast<SolveFlags *>(flags);
    int *tdone = flags + 4;
    int *cnt = tdone + nblk + 1;
    int *bcnt = cnt + (nblk + 1) * nblk;
    double *z = Z + 16;  // z(4:), 4 per row; y' then x' overwrite it
    if (blockIdx.x == 0) solve_chain(A, m, z, status, F, tdone, cnt, bcnt, limit_ns, sm);
    else solve_others(A, m, z, status, F, tdone, cnt, bcnt, limit_ns, sm);
}

constexpr size_t kSolveSmem = sizeof(double) * (3 * kNB * (kNB + 1) + 3 * kNB);

// 4c. c = H1 H2 H3 H4 [0; w]  (Z rows 0..3 are replaced by zeros)
__global__ void k_apply_q(int n, const double *V, const double *tau, const double *Z, double *C)
{
    __shared__ double sh[32];
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int c = 0; c < 4; ++c) C[i * 4 + c] = i < 4 ? 0.0 : Z[i * 4 + c];
    __syncthreads();
    for (int k = 3; k >= 0; --k) {
        for (int c = 0; c < 4; ++c) {
            double d = 0.0;
            for (int i = threadIdx.x; i < n; i += blockDim.x) d += V[i * 4 + k] * C[i * 4 + c];
            d = tau[k] * block_sum(d, sh);
            for (int i = threadIdx.x; i < n; i += blockDim.x) C[i * 4 + c] -= d * V[i * 4 + k];
            __syncthreads();
        }
    }
}

// 4d. d = R^-1 (Q' (Y - K c))(0:4); KC = K c precomputed.
__global__ void k_finish_d(int n, const double *V, const double *tau, const double *R, const double *Y, double *KC,
                           double *d_out)
{
    __shared__ double sh[32];
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int c = 0; c < 4; ++c) KC[i * 4 + c] = Y[i * 4 + c] - KC[i * 4 + c];
    __syncthreads();
    for (int k = 0; k < 4; ++k) {
        for (int c = 0; c < 4; ++c) {
            double d = 0.0;
            for (int i = threadIdx.x; i < n; i += blockDim.x) d += V[i * 4 + k] * KC[i * 4 + c];
            d = tau[k] * block_sum(d, sh);
            for (int i = threadIdx.x; i < n; i += blockDim.x) KC[i * 4 + c] -= d * V[i * 4 + k];
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        for (int c = 0; c < 4; ++c)
            for (int a = 3; a >= 0; --a) {
                double s = KC[a * 4 + c];
                for (int b = a + 1; b < 4; ++b) s -= R[a * 4 + b] * d_out[b * 4 + c];
                d_out[a * 4 + c] = s / R[a * 4 + a];
            }
    }
}

// 5. FP32 evaluation arrays: centres relative to the origin o, and the
// negated non-affine coefficients (-c_x, -c_y, -c_z, 0).
__global__ void k_eval_arrays(int n, const double *ctr, const double *C, double ox, double oy, double oz,
                              float4 *ctr32, float4 *coef32)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ctr32[i] = make_float4((float)(ctr[3 * i] - ox), (float)(ctr[3 * i + 1] - oy), (float)(ctr[3 * i + 2] - oz), 0.f);
    coef32[i] = make_float4((float)(-C[4 * i + 1]), (float)(-C[4 * i + 2]), (float)(-C[4 * i + 3]), 0.f);
}

// ----------------------------------------------------------- affine DLT

__global__ void k_affine_fit(const double *tar, const double *sub, int n, double *out, int *status)
{
    __shared__ double sh[32];
    __shared__ double ata[13][13];
    __shared__ double nrm[2][4];  // scale, cx, cy, cz for A (tar) and B (sub)
    for (int s = 0; s < 2; ++s) {
        const double *p = s == 0 ? tar : sub;
        double cx = 0, cy = 0, cz = 0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) { cx += p[3 * i]; cy += p[3 * i + 1]; cz += p[3 * i + 2]; }
        cx = block_sum(cx, sh) / n;
        cy = block_sum(cy, sh) / n;
        cz = block_sum(cz, sh) / n;
        double dsum = 0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double dx = p[3 * i] - cx, dy = p[3 * i + 1] - cy, dz = p[3 * i + 2] - cz;
            dsum += sqrt(dx * dx + dy * dy + dz * dz);
        }
        dsum = block_sum(dsum, sh) / n;
        if (threadIdx.x == 0) { nrm[s][0] = 1.0 / dsum; nrm[s][1] = cx; nrm[s][2] = cy; nrm[s][3] = cz; }
        __syncthreads();
    }
    // normal matrix of the 3n x 13 DLT system, row block per point:
    // [a 1 0 0 -bx], [0 a 1 0 -by], [0 0 a 1 -bz] with a = (ax, ay, az)
    for (int e = 0; e < 169; ++e) {
        const int r = e / 13, c = e % 13;
        if (c < r) continue;
        double acc = 0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double a[3], b[3];
            for (int q = 0; q < 3; ++q) {
                a[q] = (tar[3 * i + q] - nrm[0][1 + q]) * nrm[0][0];
                b[q] = (sub[3 * i + q] - nrm[1][1 + q]) * nrm[1][0];
            }
            for (int rb = 0; rb < 3; ++rb) {
                double row[13] = {0};
                row[rb * 4 + 0] = a[0]; row[rb * 4 + 1] = a[1]; row[rb * 4 + 2] = a[2]; row[rb * 4 + 3] = 1.0;
                row[12] = -b[rb];
                acc += row[r] * row[c];
            }
        }
        acc = block_sum(acc, sh);
        if (threadIdx.x == 0) { ata[r][c] = acc; ata[c][r] = acc; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double Vm[13][13];
        for (int i = 0; i < 13; ++i)
            for (int j = 0; j < 13; ++j) Vm[i][j] = i == j ? 1.0 : 0.0;
        for (int sweep = 0; sweep < 100; ++sweep) {
            double off = 0, diag = 0;
            for (int p = 0; p < 13; ++p) {
                diag += ata[p][p] * ata[p][p];
                for (int q = p + 1; q < 13; ++q) off += ata[p][q] * ata[p][q];
            }
            if (off <= 1e-30 * diag) break;
            for (int p = 0; p < 12; ++p)
                for (int q = p + 1; q < 13; ++q) {
                    double apq = ata[p][q];
                    if (fabs(apq) < 1e-300) continue;
                    double theta = (ata[q][q] - ata[p][p]) / (2.0 * apq);
                    double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                    for (int k = 0; k < 13; ++k) {
                        double akp = ata[k][p], akq = ata[k][q];
                        ata[k][p] = cs * akp - sn * akq;
                        ata[k][q] = sn * akp + cs * akq;
                    }
                    for (int k = 0; k < 13; ++k) {
                        double apk = ata[p][k], aqk = ata[q][k];
                        ata[p][k] = cs * apk - sn * aqk;
                        ata[q][k] = sn * apk + cs * aqk;
                    }
                    for (int k = 0; k < 13; ++k) {
                        double vkp = Vm[k][p], vkq = Vm[k][q];
                        Vm[k][p] = cs * vkp - sn * vkq;
                        Vm[k][q] = sn * vkp + cs * vkq;
                    }
                }
        }
        int best = 0;
        for (int p = 1; p < 13; ++p)
            if (ata[p][p] < ata[best][best]) best = p;
        double h[13];
        for (int i = 0; i < 13; ++i) h[i] = Vm[i][best];
        if (h[12] == 0.0) {
            atomicOr(status, kStSingularX);
            return;
        }
        for (int i = 0; i < 13; ++i) h[i] /= h[12];
        // T = NB^-1 H NA with N = [s I, -s c; 0 1]:  NB^-1 = [I/sB, cB; 0 1]
        const double sA = nrm[0][0], sB = nrm[1][0];
        double H[3][4];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) H[r][c] = h[r * 4 + c];
        for (int r = 0; r < 3; ++r) {
            // (H NA)(r,:) = [sA H(r,0:3), H(r,3) - sA H(r,0:3).cA]
            double lin[3], tr = H[r][3];
            for (int c = 0; c < 3; ++c) {
                lin[c] = sA * H[r][c];
                tr -= sA * H[r][c] * nrm[0][1 + c];
            }
            for (int c = 0; c < 3; ++c) out[r * 4 + c] = lin[c] / sB;
            out[r * 4 + 3] = tr / sB + nrm[1][1 + r];
        }
        out[12] = 0; out[13] = 0; out[14] = 0; out[15] = 1;
    }
}

struct DevBuf {
    tw_ctx *ctx = nullptr;
    void *p = nullptr;
    size_t bytes = 0;
    ~DevBuf() { if (p) dfree(ctx, p, bytes); }
};

struct StreamBuf {
    tw_ctx *ctx = nullptr;
    cudaStream_t st = nullptr;
    void *p = nullptr;
    size_t bytes = 0;
    ~StreamBuf() { if (p) dfree_on(ctx, p, bytes, st); }
};

}  // namespace

tw_status solve_tps_device(tw_ctx *ctx, const double *h_ctr, const double *h_val, int n, double lambda,
                           double *d_c_out, double *d_d_out, int *d_status_out, double *h_d_out, const double o[3],
                           float4 *ctr32_out, float4 *coef32_out, cudaStream_t st, double *h_stage)
{
    const int m = n - 4;
    // workspace: ctr 3n, Y 4n, Xw 4n, V 4n, P 4n, W 4n, Z 4n, KC 4n, tau 4, R 16, d 16, status
    // ctr 3n, Y/Xw/V/P/W/Z/KC 4n each, tau 4, R 16, then the solve kernel's
    // dependency counters (ints)
    const int nblk = m > 0 ? (m + kNB - 1) / kNB : 0;
    const size_t nflags = 4 + (size_t)(nblk + 1) + (size_t)(nblk + 1) * nblk + (size_t)nblk;
    const size_t small = 3 * (size_t)n + 7 * 4 * (size_t)n + 4 + 16 + (nflags + 1) / 2;
    // stream-ordered workspace on `st`, returned to the pool on `st` when this
    // function exits (after the final wait, or with the error)
    StreamBuf ws{ctx, st}, abuf{ctx, st};
    ws.bytes = small * sizeof(double);
    TW_TRY(dmalloc_on(ctx, &ws.p, ws.bytes, st));
    double *base = static_cast<double *>(ws.p);
    double *d_ctr = base;
    double *d_Y = d_ctr + 3 * (size_t)n;
    double *d_Xw = d_Y + 4 * (size_t)n;
    double *d_V = d_Xw + 4 * (size_t)n;
    double *d_P = d_V + 4 * (size_t)n;
    double *d_W = d_P + 4 * (size_t)n;
    double *d_Z = d_W + 4 * (size_t)n;
    double *d_KC = d_Z + 4 * (size_t)n;
    double *d_tau = d_KC + 4 * (size_t)n;
    double *d_R = d_tau + 4;
    double *d_d = d_d_out;
    int *d_status = d_status_out;
    int *d_flags = reinterpret_cast<int *>(d_R + 16);
    if (m > 0) {
        abuf.bytes = (size_t)(m + 4) * m * sizeof(double);
        TW_TRY(dmalloc_on(ctx, &abuf.p, abuf.bytes, st));
    }
    double *d_A = static_cast<double *>(abuf.p);

    std::vector<double> hY(4 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        hY[4 * i + 0] = 1.0;
        hY[4 * i + 1] = h_val[3 * i + 0];
        hY[4 * i + 2] = h_val[3 * i + 1];
        hY[4 * i + 3] = h_val[3 * i + 2];
    }
    if (h_stage) {
        std::memcpy(h_stage, h_ctr, sizeof(double) * 3 * n);
        std::memcpy(h_stage + 3 * (size_t)n, hY.data(), sizeof(double) * 4 * n);
        TW_CUDA_TRY(cudaMemcpyAsync(d_ctr, h_stage, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
        TW_CUDA_TRY(cudaMemcpyAsync(d_Y, h_stage + 3 * (size_t)n, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, st));
    } else {
        TW_TRY(upload(ctx, d_ctr, h_ctr, sizeof(double) * 3 * n, st));
        TW_TRY(upload(ctx, d_Y, hY.data(), sizeof(double) * 4 * n, st));
    }
    TW_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    TW_CUDA_TRY(cudaMemsetAsync(d_d, 0, sizeof(double) * 16, st));

    uint64_t nl = 0;
    k_qr<<<1, kRedThreads, 0, st>>>(d_ctr, n, d_Xw, d_V, d_tau, d_R, d_status);
    ++nl;
    const int warps_per_block = 8;
    const unsigned kgrid = (unsigned)((n + warps_per_block - 1) / warps_per_block);
    k_kmul<<<kgrid, 32 * warps_per_block, 0, st>>>(d_ctr, n, d_V, d_P);
    k_wvec<<<1, kRedThreads, 0, st>>>(n, d_V, d_tau, d_P, d_W, d_Y, d_Z);
    nl += 2;
    if (m > 0) {
        dim3 b(32, 8), g((m + 31) / 32, (m + 4 + 7) / 8);
        k_fill_a<<<g, b, 0, st>>>(d_ctr, n, d_V, d_W, d_Z, lambda, d_A);
        ++nl;
        TW_CUDA_TRY(cudaFuncSetAttribute(k_chol_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSolveSmem));
        int per_sm = 0;
        TW_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_chol_solve, kSolveThreads, kSolveSmem));
        if (per_sm < 1) return fail(ctx, TW_ERR_CUDA, "solve kernel does not fit on an SM");
        int grid = ctx->sm_count;
        TW_CUDA_TRY(cudaMemsetAsync(d_flags, 0, sizeof(int) * nflags, st));
        unsigned long long limit_ns = ctx->solve_barrier_ns.load();
        void *args[] = {(void *)&d_A, (void *)&m, (void *)&d_Z, (void *)&d_status, (void *)&d_flags, (void *)&limit_ns};
        TW_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)k_chol_solve, dim3(grid), dim3(kSolveThreads), args,
                                                kSolveSmem, st));
        ++nl;
    }
    k_apply_q<<<1, kRedThreads, 0, st>>>(n, d_V, d_tau, d_Z, d_c_out);
    k_kmul<<<kgrid, 32 * warps_per_block, 0, st>>>(d_ctr, n, d_c_out, d_KC);
    k_finish_d<<<1, kRedThreads, 0, st>>>(n, d_V, d_tau, d_R, d_Y, d_KC, d_d);
    nl += 3;
    if (ctr32_out && coef32_out) {
        k_eval_arrays<<<(n + 255) / 256, 256, 0, st>>>(n, d_ctr, d_c_out, o[0], o[1], o[2], ctr32_out, coef32_out);
        ++nl;
    }
    TW_CUDA_TRY(cudaGetLastError());
    count_launch(ctx, nl);
    if (!h_d_out) return TW_OK;  // the caller reads the status later
    TW_CUDA_TRY(cudaMemcpyAsync(h_d_out, d_d, sizeof(double) * 16, cudaMemcpyDeviceToHost, st));
    return solve_status(ctx, d_status, st);
}

tw_status solve_status(tw_ctx *ctx, const int *d_status, cudaStream_t st)
{
    int status = 0;
    TW_CUDA_TRY(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    TW_CUDA_TRY(cudaStreamSynchronize(st));
    if (status & kStSingularX)
        return fail(ctx, TW_ERR_SINGULAR, "TPS centres are degenerate: [1 s] is rank deficient (coplanar or < 4 distinct points)");
    if (status & kStTimeout)
        return fail(ctx, TW_ERR_TIMEOUT, "TPS solve: a wait on another block of the solve timed out");
    if (status & kStNotSPD)
        return fail(ctx, TW_ERR_SINGULAR, "projected TPS system is not positive definite");
    return TW_OK;
}

tw_status fit_affine_device(tw_ctx *ctx, const double *h_tar, const double *h_sub, int n, double M[16],
                            cudaStream_t st)
{
    DevBuf ws{ctx};
    ws.bytes = sizeof(double) * (6 * (size_t)n + 16 + 2);
    TW_TRY(dmalloc(ctx, &ws.p, ws.bytes));
    double *d_tar = static_cast<double *>(ws.p);
    double *d_sub = d_tar + 3 * (size_t)n;
    double *d_out = d_sub + 3 * (size_t)n;
    int *d_status = reinterpret_cast<int *>(d_out + 16);
    TW_CUDA_TRY(cudaMemcpyAsync(d_tar, h_tar, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    TW_CUDA_TRY(cudaMemcpyAsync(d_sub, h_sub, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    TW_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    k_affine_fit<<<1, 256, 0, st>>>(d_tar, d_sub, n, d_out, d_status);
    TW_CUDA_TRY(cudaGetLastError());
    count_launch(ctx, 1);
    int status = 0;
    TW_CUDA_TRY(cudaMemcpyAsync(M, d_out, sizeof(double) * 16, cudaMemcpyDeviceToHost, st));
    TW_CUDA_TRY(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    TW_CUDA_TRY(cudaStreamSynchronize(st));
    if (status) return fail(ctx, TW_ERR_SINGULAR, "affine DLT is degenerate (h13 = 0)");
    return TW_OK;
}

cudaError_t launch_affine_fit(const double *d_tar, const double *d_sub, int n, double *d_out, int *d_status,
                              cudaStream_t st)
{
    k_affine_fit<<<1, 256, 0, st>>>(d_tar, d_sub, n, d_out, d_status);
    return cudaGetLastError();
}

}  // namespace tw
