// pcg.cu -- Jacobi-preconditioned CG on the device for sm_100a.
//
// Reference: conjugate_gradient::solve (src/solver/linear/linear_solver.cpp:67-109), which runs
// Eigen's ConjugateGradient<Lower|Upper> with the diagonal preconditioner, x0 = 0 and the stop
// test ||r||^2 < max(tol^2 ||b||^2, DBL_MIN), and the reference's GPU variant
// conjugate_gradient_cuda::solve (conjugate_gradient_cuda.cpp:72-192, cuSPARSE csrmv + cuBLAS
// + diagonal_matrix_vector_product.cu) which copies K to the device on every solve and reads 3
// dot products back to the host per iteration.
//
// Here K stays resident in HBM and every scalar stays on the device.  One iteration is three
// kernels:
//   k_spmv  : q = A p over the 3x3 block rows (a few lanes per block row, several rows per
//             warp in flight), fused with the p.q reduction; the last block to finish forms
//             alpha = (r.z)/(p.q);
//   k_xr    : x += alpha p, r -= alpha q, fused with r.r and r.z (z = D^-1 r); the last block
//             applies the stop test, beta and the iteration count;
//   k_p     : p = D^-1 r + beta p.
// Reductions are per-block partials summed in a fixed order by the last block (deterministic,
// no spin waits).  Kernels return at once after `done` is set, so whole blocks of iterations are
// enqueued (optionally as one CUDA graph) and the host reads the flag once per block.
// Rows of active Dirichlet DOFs are skipped (q = 0): with b = 0 there, r, z, p stay exactly 0 on
// them, so this equals neon's zeroing of those rows and columns (static_matrix.hpp:279-320).
#include <cfloat>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <vector>

#include "nb2_internal.cuh"

namespace nb2 {

int reduction_blocks(const nb2_ctx*) { return 148 * 4; }

template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) {
    return __ldcs(p);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV doubles into partials[blockIdx*NV + j]; returns true in the last block
// (after which s_red holds nothing useful and the caller reduces partials itself).
template <int NV>
__device__ bool block_partials(double (&v)[NV], double* partials, unsigned int* counter) {
    __shared__ double red[NV][kRedThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double t = warp_sum(v[j]);
        if (lane == 0) red[j][wid] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[j][w];
            partials[blockIdx.x * NV + j] = t;
        }
        __threadfence();
        unsigned int ticket = atomicAdd(counter, 1u);
        last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    return last;
}

// Fixed-order sum of partials[b*NV + j] over b (called by the whole last block).
template <int NV>
__device__ void final_sum(const double* partials, double (&out)[NV]) {
    __shared__ double red[NV][kRedThreads];
    __threadfence();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double t = 0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
            t += *((volatile const double*)&partials[b * NV + j]);
        red[j][threadIdx.x] = t;
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
#pragma unroll
            for (int j = 0; j < NV; ++j) red[j][threadIdx.x] += red[j][threadIdx.x + s];
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < NV; ++j) out[j] = red[j][0];
}

// ---------------------------------------------------------------------------------------
// matrices
// ---------------------------------------------------------------------------------------
template <typename V>
struct Bsr {
    const int* brp;
    const int* bcol;
    const V* val;
    int rows;  // block rows
};

struct Csr {
    const int* rp;
    const int* ci;
    const double* val;
    int rows;
};

// y[3a+r] for r = 0..2 of block row a, reduced across the warp (all lanes get the sums).
// A row of a hex8 mesh holds up to 27 blocks = 243 values: the first 256 values are loaded in one
// batch of 8 independent loads per lane (values, then their block columns, then the x entries),
// so a warp keeps a whole row in flight instead of one 32-value slice per round trip.
template <typename V, typename X, typename Acc>
__device__ __forceinline__ void bsr_row(const Bsr<V>& A, const X* __restrict__ x, int a, int lane,
                                        Acc& y0, Acc& y1, Acc& y2) {
    const int b0 = __ldg(A.brp + a);
    const int nval = 9 * (__ldg(A.brp + a + 1) - b0);
    const V* vals = A.val + 9ll * b0;
    const int* cols = A.bcol + b0;
    Acc a0 = 0, a1 = 0, a2 = 0;
    constexpr int U = 8;
    V v[U];
    int c[U];
#pragma unroll
    for (int t = 0; t < U; ++t) {
        const int idx = lane + 32 * t;
        const bool ok = idx < nval;
        v[t] = ok ? ld_stream(vals + idx) : (V)0;
        c[t] = ok ? __ldg(cols + idx / 9) : 0;
    }
#pragma unroll
    for (int t = 0; t < U; ++t) {
        const int idx = lane + 32 * t;
        const int e = idx % 9;
        const int r = e / 3;
        const int cc = e - 3 * r;
        const Acc prod = (Acc)v[t] * (Acc)x[3ll * c[t] + cc];
        a0 += (r == 0) ? prod : (Acc)0;
        a1 += (r == 1) ? prod : (Acc)0;
        a2 += (r == 2) ? prod : (Acc)0;
    }
    for (int idx = lane + 32 * U; idx < nval; idx += 32) {  // rows with more than 28 blocks
        const int k = idx / 9;
        const int e = idx - 9 * k;
        const int r = e / 3;
        const int cc = e - 3 * r;
        const Acc prod = (Acc)ld_stream(vals + idx) * (Acc)x[3ll * __ldg(cols + k) + cc];
        a0 += (r == 0) ? prod : (Acc)0;
        a1 += (r == 1) ? prod : (Acc)0;
        a2 += (r == 2) ? prod : (Acc)0;
    }
    y0 = warp_sum(a0);
    y1 = warp_sum(a1);
    y2 = warp_sum(a2);
}

// ---------------------------------------------------------------------------------------
// CG kernels (BSR)
// ---------------------------------------------------------------------------------------
// q = A p with LPR lanes per 3x3 block row: a warp keeps 32/LPR rows in flight; lane l of a row
// walks its blocks l, l+LPR, ... (9 values, the block column, 3 gathered p entries) and the three
// row sums are reduced over the LPR lanes with shuffles.  Plain loads with many independent rows
// per SM stream the matrix at ~80% of HBM bandwidth (hex8 rows: 27 blocks, tet4: ~15), where a
// whole warp per row or a shared-memory staging pipeline left it latency-bound.  Fused with the
// p.q reduction; the last block forms alpha = (r.z)/(p.q).
template <typename V, typename X, int LPR>
__global__ void __launch_bounds__(kRedThreads) k_spmv(Bsr<V> A, const X* __restrict__ p,
                                                      X* __restrict__ q,
                                                      const unsigned char* __restrict__ mask,
                                                      CgScalars* s, double* partials) {
    if (s->done) return;
    constexpr int RPW = 32 / LPR;
    const int lane = threadIdx.x & 31, sub = lane / LPR, sl = lane % LPR;
    const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    double dot[1] = {0.0};
    for (long long a0 = gw * RPW; a0 < A.rows; a0 += nw * RPW) {
        const long long a = a0 + sub;
        X y0 = 0, y1 = 0, y2 = 0;
        if (a < A.rows) {
            const int b0 = A.brp[a], b1 = A.brp[a + 1];
            for (int k = b0 + sl; k < b1; k += LPR) {
                const long long col = A.bcol[k];
                const X x0 = p[3 * col], x1 = p[3 * col + 1], x2 = p[3 * col + 2];
                const V* blk = A.val + 9ll * k;
                y0 += (X)blk[0] * x0 + (X)blk[1] * x1 + (X)blk[2] * x2;
                y1 += (X)blk[3] * x0 + (X)blk[4] * x1 + (X)blk[5] * x2;
                y2 += (X)blk[6] * x0 + (X)blk[7] * x1 + (X)blk[8] * x2;
            }
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, o);
            y1 += __shfl_xor_sync(0xffffffffu, y1, o);
            y2 += __shfl_xor_sync(0xffffffffu, y2, o);
        }
        if (a < A.rows && sl < 3) {
            const long long i = 3 * a + sl;
            X y = sl == 0 ? y0 : (sl == 1 ? y1 : y2);
            if (mask && mask[i]) y = (X)0;
            q[i] = y;
            dot[0] += (double)p[i] * (double)y;
        }
    }
    if (block_partials<1>(dot, partials, &s->counter[0])) {
        double tot[1];
        final_sum<1>(partials, tot);
        if (threadIdx.x == 0) {
            s->pq = tot[0];
            s->alpha = s->abs_new / tot[0];
            // Eigen's CG carries on through p.Ap <= 0 (an indefinite tangent); only a
            // non-finite step size is a failure (neon: FE_INVALID -> computational_error)
            if (!isfinite(s->alpha)) {
                s->status = NB2_E_NAN;
                s->done = 1;
            }
            s->counter[0] = 0;
        }
    }
}

// lanes per block row of the PCG SpMV: 4 for FP64 and FP32 values (C3 on B200: FP64 0.44 ms,
// FP32 0.26 ms per iteration; 8 or 16 lanes were slower for both)
template <typename V>
constexpr int spmv_lanes() {
    return 4;
}

// 16-byte vector view of the CG vectors (float4 / double2): the update kernels move W values
// per load and store when every vector is 16-byte aligned (device allocations are; a caller's
// buffers may not be, then the scalar loop does all of it)
template <typename X>
struct Vec16;
template <>
struct Vec16<float> {
    using T = float4;
    static constexpr int W = 4;
};
template <>
struct Vec16<double> {
    using T = double2;
    static constexpr int W = 2;
};

__device__ __forceinline__ bool aligned16(const void* a, const void* b, const void* c,
                                          const void* d, const void* e) {
    return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) |
             reinterpret_cast<uintptr_t>(c) | reinterpret_cast<uintptr_t>(d) |
             reinterpret_cast<uintptr_t>(e)) & 15) == 0;
}

template <typename X>
__device__ __forceinline__ void xr_one(X& x, X& r, X p, X q, X inv, X alpha, double (&acc)[2]) {
    x += alpha * p;
    const X ri = r - alpha * q;
    r = ri;
    acc[0] += (double)ri * (double)ri;
    acc[1] += (double)ri * (double)(inv * ri);
}

template <typename X>
__global__ void __launch_bounds__(kRedThreads) k_xr(long long n, X* __restrict__ x,
                                                    X* __restrict__ r, const X* __restrict__ p,
                                                    const X* __restrict__ q,
                                                    const X* __restrict__ inv, CgScalars* s,
                                                    double* partials) {
    if (s->done) return;
    using V = typename Vec16<X>::T;
    constexpr int W = Vec16<X>::W;
    const X alpha = (X)s->alpha;
    double acc[2] = {0.0, 0.0};
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long st = (long long)gridDim.x * blockDim.x;
    const long long nv = aligned16(x, r, p, q, inv) ? n / W : 0;
    for (long long j = t0; j < nv; j += st) {
        X xv[W], rv[W], pv[W], qv[W], iv[W];
        *reinterpret_cast<V*>(xv) = reinterpret_cast<const V*>(x)[j];
        *reinterpret_cast<V*>(rv) = reinterpret_cast<const V*>(r)[j];
        *reinterpret_cast<V*>(pv) = reinterpret_cast<const V*>(p)[j];
        *reinterpret_cast<V*>(qv) = reinterpret_cast<const V*>(q)[j];
        *reinterpret_cast<V*>(iv) = reinterpret_cast<const V*>(inv)[j];
#pragma unroll
        for (int w = 0; w < W; ++w) xr_one(xv[w], rv[w], pv[w], qv[w], iv[w], alpha, acc);
        reinterpret_cast<V*>(x)[j] = *reinterpret_cast<V*>(xv);
        reinterpret_cast<V*>(r)[j] = *reinterpret_cast<V*>(rv);
    }
    for (long long i = nv * W + t0; i < n; i += st) xr_one(x[i], r[i], p[i], q[i], inv[i], alpha, acc);
    if (block_partials<2>(acc, partials, &s->counter[1])) {
        double tot[2];
        final_sum<2>(partials, tot);
        if (threadIdx.x == 0) {
            s->rr = tot[0];
            if (tot[0] < s->threshold) {
                s->done = 1;
            } else if (tot[0] > s->rr_cap) {
                s->done = 1;
                s->status = NB2_E_CG_BREAKDOWN;
            } else {
                s->beta = tot[1] / s->abs_new;
                s->abs_new = tot[1];
                s->rz = tot[1];
                s->iterations += 1;
                if (s->iterations >= s->max_iterations) {
                    s->done = 1;
                    s->status = NB2_E_CG_MAXIT;
                }
            }
            if (!isfinite(tot[0])) {
                s->done = 1;
                s->status = NB2_E_NAN;
            }
            s->counter[1] = 0;
        }
    }
}

template <typename X>
__global__ void __launch_bounds__(kRedThreads) k_p(long long n, X* __restrict__ p,
                                                   const X* __restrict__ r,
                                                   const X* __restrict__ inv, const CgScalars* s) {
    if (s->done) return;
    using V = typename Vec16<X>::T;
    constexpr int W = Vec16<X>::W;
    const X beta = (X)s->beta;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long st = (long long)gridDim.x * blockDim.x;
    const long long nv = aligned16(p, r, inv, p, r) ? n / W : 0;
    for (long long j = t0; j < nv; j += st) {
        X pv[W], rv[W], iv[W];
        *reinterpret_cast<V*>(pv) = reinterpret_cast<const V*>(p)[j];
        *reinterpret_cast<V*>(rv) = reinterpret_cast<const V*>(r)[j];
        *reinterpret_cast<V*>(iv) = reinterpret_cast<const V*>(inv)[j];
#pragma unroll
        for (int w = 0; w < W; ++w) pv[w] = iv[w] * rv[w] + beta * pv[w];
        reinterpret_cast<V*>(p)[j] = *reinterpret_cast<V*>(pv);
    }
    for (long long i = nv * W + t0; i < n; i += st) p[i] = inv[i] * r[i] + beta * p[i];
}

// x = 0, r = b (as X), p = D^-1 r; rhs_norm2, r.r, r.p; threshold and early exits.
template <typename X>
__global__ void __launch_bounds__(kRedThreads) k_init(long long n, const double* __restrict__ b,
                                                      X* __restrict__ x, X* __restrict__ r,
                                                      X* __restrict__ p,
                                                      const X* __restrict__ inv, CgScalars* s,
                                                      double* partials, double tol) {
    double acc[3] = {0, 0, 0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        X bi = (X)b[i];
        x[i] = (X)0;
        r[i] = bi;
        X pi = inv[i] * bi;
        p[i] = pi;
        acc[0] += b[i] * b[i];
        acc[1] += (double)bi * (double)bi;
        acc[2] += (double)bi * (double)pi;
    }
    if (block_partials<3>(acc, partials, &s->counter[2])) {
        double tot[3];
        final_sum<3>(partials, tot);
        if (threadIdx.x == 0) {
            s->rhs_norm2 = tot[0];
            s->threshold = fmax(tol * tol * tot[0], DBL_MIN);
            s->rr = tot[1];
            s->abs_new = tot[2];
            s->rz = tot[2];
            s->rr_cap = INFINITY;
            s->iterations = 0;
            s->status = 0;
            s->done = 0;
            if (tot[0] == 0.0) {
                s->done = 1;
                s->rr = 0.0;
            } else if (tot[1] < s->threshold) {
                s->done = 1;
            }
            s->counter[2] = 0;
        }
    }
}

// Jacobi inverse diagonal of a block matrix: 1/K_ii, or 1 for a zero diagonal (Eigen's
// DiagonalPreconditioner).
template <typename V, typename X>
__global__ void k_invdiag(Bsr<V> A, X* __restrict__ inv) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A.rows) return;
    int lo = A.brp[a], hi = A.brp[a + 1] - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (A.bcol[mid] < a)
            lo = mid + 1;
        else
            hi = mid;
    }
    // a node that no element references has an empty row: its diagonal is 0 (inverse 1)
    const bool has = lo < A.brp[a + 1] && A.bcol[lo] == a;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        V d = has ? A.val[9ll * lo + 4 * r] : (V)0;
        inv[3ll * a + r] = (d != (V)0) ? (X)(1.0 / (double)d) : (X)1;
    }
}

template <typename X>
__global__ void k_copy_out(long long n, const X* __restrict__ src, double* __restrict__ dst) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

// ---------------------------------------------------------------------------------------
// generic CSR (drop-in linear_solver on a caller matrix)
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kRedThreads) k_csr_spmv(Csr A, const double* __restrict__ p,
                                                          double* __restrict__ q, CgScalars* s,
                                                          double* partials) {
    if (s->done) return;
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    double dot[1] = {0.0};
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < A.rows; i += warps) {
        double acc = 0;
        for (int k = A.rp[i] + lane; k < A.rp[i + 1]; k += 32) acc += A.val[k] * p[A.ci[k]];
        acc = warp_sum(acc);
        if (lane == 0) {
            q[i] = acc;
            dot[0] += p[i] * acc;
        }
    }
    if (block_partials<1>(dot, partials, &s->counter[0])) {
        double tot[1];
        final_sum<1>(partials, tot);
        if (threadIdx.x == 0) {
            s->pq = tot[0];
            s->alpha = s->abs_new / tot[0];
            if (!isfinite(s->alpha)) {
                s->status = NB2_E_NAN;
                s->done = 1;
            }
            s->counter[0] = 0;
        }
    }
}

__global__ void k_csr_invdiag(Csr A, double* inv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.rows) return;
    double v = 1.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if (A.ci[k] == i) {
            if (A.val[k] != 0.0) v = 1.0 / A.val[k];
            break;
        }
    inv[i] = v;
}

// ---------------------------------------------------------------------------------------
// norms and helpers
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kRedThreads) k_norms(long long n, const double* a,
                                                       const double* b, const double* c,
                                                       const double* d, const double* e,
                                                       double* partials, unsigned int* counter,
                                                       double* out) {
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        acc[0] += a[i] * a[i];
        acc[1] += b[i] * b[i];
        acc[2] += c[i] * c[i];
        acc[3] += d[i] * d[i];
        acc[4] += e[i] * e[i];
    }
    if (block_partials<5>(acc, partials, counter)) {
        double tot[5];
        final_sum<5>(partials, tot);
        if (threadIdx.x == 0) {
            for (int j = 0; j < 5; ++j) out[j] = sqrt(tot[j]);
            *counter = 0;
        }
    }
}

template <typename V>
__global__ void __launch_bounds__(kRedThreads) k_bsr_apply(Bsr<V> A, const double* __restrict__ x,
                                                           double* __restrict__ y,
                                                           const unsigned char* __restrict__ mask) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); a < A.rows; a += warps) {
        double y0, y1, y2;
        bsr_row<V, double, double>(A, x, a, lane, y0, y1, y2);
        if (lane < 3) {
            long long i = 3ll * a + lane;
            double v = lane == 0 ? y0 : (lane == 1 ? y1 : y2);
            if (mask && mask[i]) v = 0.0;
            y[i] = v;
        }
    }
}

// ---------------------------------------------------------------------------------------
// matrix-free FP32 operator: node-ordered gather of the per-element products
// ---------------------------------------------------------------------------------------
// q = sum over the node's element slots of ye (masked rows 0), p.q -> alpha (as k_spmv).  nadj
// holds each slot's position in ye's per-node planes, so neighbouring nodes read neighbouring
// elements' entries of one plane (coalesced)
template <typename X>
__global__ void __launch_bounds__(kRedThreads) k_mf_gather(int N, const int* __restrict__ nptr,
                                                           const int* __restrict__ nadj,
                                                           const float* __restrict__ ye,
                                                           const X* __restrict__ p,
                                                           X* __restrict__ q,
                                                           const unsigned char* __restrict__ mask,
                                                           CgScalars* s, double* partials) {
    if (s->done) return;
    double dot[1] = {0.0};
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < N; a += gridDim.x * blockDim.x) {
        float y0 = 0.0f, y1 = 0.0f, y2 = 0.0f;
        const int k1 = nptr[a + 1];
#pragma unroll 4
        for (int k = nptr[a]; k < k1; ++k) {
            const long long j = 3ll * nadj[k];
            y0 += ye[j];
            y1 += ye[j + 1];
            y2 += ye[j + 2];
        }
        const float y[3] = {y0, y1, y2};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const long long i = 3ll * a + c;
            const X v = mask[i] ? (X)0 : (X)y[c];
            q[i] = v;
            dot[0] += (double)p[i] * (double)v;
        }
    }
    if (block_partials<1>(dot, partials, &s->counter[0])) {
        double tot[1];
        final_sum<1>(partials, tot);
        if (threadIdx.x == 0) {
            s->pq = tot[0];
            s->alpha = s->abs_new / tot[0];
            if (!isfinite(s->alpha)) {
                s->status = NB2_E_NAN;
                s->done = 1;
            }
            s->counter[0] = 0;
        }
    }
}

// y = sum over the node's element slots of ye (no mask, no reduction)
__global__ void k_mf_sum(int N, const int* __restrict__ nptr, const int* __restrict__ nadj,
                         const float* __restrict__ ye, double* __restrict__ y) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    float s[3] = {0.0f, 0.0f, 0.0f};
    for (int k = nptr[a]; k < nptr[a + 1]; ++k) {
        const long long j = 3ll * nadj[k];
        s[0] += ye[j];
        s[1] += ye[j + 1];
        s[2] += ye[j + 2];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) y[3ll * a + c] = (double)s[c];
}

__global__ void k_to_float(long long n, const double* __restrict__ a, float* __restrict__ b) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// Jacobi inverse from the per-element diagonal contributions (1 for a zero diagonal)
__global__ void k_mf_diag(int N, const int* __restrict__ nptr, const int* __restrict__ nadj,
                          const float* __restrict__ de, float* __restrict__ inv) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    double d[3] = {0.0, 0.0, 0.0};
    for (int k = nptr[a]; k < nptr[a + 1]; ++k) {
        const long long j = 3ll * nadj[k];
        d[0] += de[j];
        d[1] += de[j + 1];
        d[2] += de[j + 2];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) inv[3ll * a + c] = d[c] != 0.0 ? (float)(1.0 / d[c]) : 1.0f;
}

// ---------------------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------------------
static int wait_scalars(nb2_ctx* c) {
    NB2_CUDA(c, cudaMemcpyAsync(c->h_cgs, c->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost,
                                c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

constexpr int kChunk = 32;

// One Jacobi-PCG on a block matrix: the captured block of kChunk iterations and the host loop
// that launches blocks until the device scalars say done.
template <typename V, typename X>
struct CgRunner {
    nb2_ctx* c;
    const V* vals;
    X *x, *r, *p, *q, *inv;
    bool use_mask, use_graphs;
    cudaGraphExec_t* cache;
    bool mf = false;  // FP32 matrix-free operator (V = X = float) instead of the assembled K
    int RB = 0;
    Bsr<V> A{};

    int setup() {
        RB = reduction_blocks(c);
        if (mf) return NB2_OK;  // the Jacobi inverse comes from the matrix-free setup
        A = Bsr<V>{c->brp, c->bcol, vals, c->N};
        k_invdiag<V, X><<<(c->N + 255) / 256, 256, 0, c->stream>>>(A, inv);
        c->launches++;
        return NB2_OK;
    }

    void enqueue(int count) {
        const unsigned char* mask = use_mask ? c->mask : nullptr;
        const long long n = c->n;
        for (int it = 0; it < count; ++it) {
            if constexpr (sizeof(X) == 4) {
                if (mf) {
                    enqueue_apply32(c, p, c->mf_ye, &c->cgs->done);
                    k_mf_gather<X><<<RB, kRedThreads, 0, c->stream>>>(
                        c->N, c->nadj_ptr, c->nadj_pl, c->mf_ye, p, q, c->mask, c->cgs, c->partials);
                    k_xr<X><<<RB, kRedThreads, 0, c->stream>>>(n, x, r, p, q, inv, c->cgs,
                                                               c->partials);
                    k_p<X><<<RB, kRedThreads, 0, c->stream>>>(n, p, r, inv, c->cgs);
                    continue;
                }
            }
            k_spmv<V, X, spmv_lanes<V>()><<<RB, kRedThreads, 0, c->stream>>>(A, p, q, mask, c->cgs,
                                                                            c->partials);
            k_xr<X><<<RB, kRedThreads, 0, c->stream>>>(n, x, r, p, q, inv, c->cgs, c->partials);
            k_p<X><<<RB, kRedThreads, 0, c->stream>>>(n, p, r, inv, c->cgs);
        }
    }

    // launch blocks of iterations until the scalars say done (bounded by maxit / kChunk + 4)
    int run(int maxit) {
        if (use_graphs && *cache == nullptr) {
            // capture one block of iterations; plain launches if the stream cannot be captured
            // (e.g. the legacy default stream)
            cudaGraph_t g = nullptr;
            if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) ==
                cudaSuccess) {
                enqueue(kChunk);
                if (cudaStreamEndCapture(c->stream, &g) == cudaSuccess && g) {
                    if (cudaGraphInstantiate(cache, g, 0) != cudaSuccess) *cache = nullptr;
                    cudaGraphDestroy(g);
                }
            }
            cudaGetLastError();
            if (*cache == nullptr) use_graphs = false;
        }
        int guard = 0;
        for (;;) {
            if (use_graphs)
                NB2_CUDA(c, cudaGraphLaunch(*cache, c->stream));
            else
                enqueue(kChunk);
            c->launches += (mf ? 4 : 3) * kChunk;
            NB2_TRY(wait_scalars(c));
            if (c->h_cgs->done) break;
            if (++guard > (maxit / kChunk) + 4) break;  // scalars say not done: cannot happen
        }
        NB2_CUDA(c, cudaGetLastError());
        return NB2_OK;
    }
};

template <typename V, typename X>
static int run_bsr_cg(nb2_ctx* c, const V* vals, X* x, X* r, X* p, X* q, X* inv, const double* b,
                      double* xout, double tol, int maxit, bool use_mask, int* iterations,
                      double* error, bool use_graphs, cudaGraphExec_t* cache) {
    CgRunner<V, X> cg{c, vals, x, r, p, q, inv, use_mask, use_graphs, cache};
    NB2_TRY(cg.setup());
    const long long n = c->n;
    k_init<X><<<cg.RB, kRedThreads, 0, c->stream>>>(n, b, x, r, p, inv, c->cgs, c->partials, tol);
    c->launches++;
    // max_iterations is read by k_xr: set it with a tiny copy
    NB2_CUDA(c, cudaMemcpyAsync(&c->cgs->max_iterations, &maxit, sizeof(int), cudaMemcpyHostToDevice,
                                c->stream));
    NB2_TRY(cg.run(maxit));
    k_copy_out<X><<<cg.RB, kRedThreads, 0, c->stream>>>(n, x, xout);
    c->launches++;
    const CgScalars& h = *c->h_cgs;
    *iterations = h.iterations;
    *error = h.rhs_norm2 > 0 ? std::sqrt(h.rr / h.rhs_norm2) : 0.0;
    if (h.status) return h.status;
    if (!h.done) return NB2_E_TIMEOUT;
    return NB2_OK;
}

// x64[i] += xs[i]; xs[i] = 0 (fold the FP32 increment into the FP64 iterate)
__global__ void k_fold(long long n, float* __restrict__ xs, double* __restrict__ x64) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        x64[i] += (double)xs[i];
        xs[i] = 0.0f;
    }
}

// r = b - y on free rows, 0 on masked rows; rs = (float) r; reduce r.r (FP64), rs.D^-1 rs
__global__ void __launch_bounds__(kRedThreads) k_true_residual(
    long long n, const double* __restrict__ b, const double* __restrict__ y,
    const unsigned char* __restrict__ mask, const float* __restrict__ inv, float* __restrict__ rs,
    CgScalars* s, double* partials, double* rr_out) {
    double acc[2] = {0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double ri = mask[i] ? 0.0 : b[i] - y[i];
        const float rf = (float)ri;
        rs[i] = rf;
        acc[0] += ri * ri;
        acc[1] += (double)rf * (double)(inv[i] * rf);
    }
    if (block_partials<2>(acc, partials, &s->counter[3])) {
        double tot[2];
        final_sum<2>(partials, tot);
        if (threadIdx.x == 0) {
            *rr_out = tot[0];
            // continue the recurrence with the replaced residual: beta = rz_new / rz_old
            s->beta = tot[1] / s->abs_new;
            s->abs_new = tot[1];
            s->rz = tot[1];
            s->rr = tot[0];
            // a cycle whose FP32 recurrence r.r grows to this multiple of the replaced one has
            // diverged (CG residual norms are not monotone: a factor 1000 in the norm)
            s->rr_cap = 1e6 * tot[0];
            s->counter[3] = 0;
        }
    }
}

// Mixed-precision PCG with reliable updates (residual replacement): the iterations run in FP32
// on K32 (FP64 dot products); whenever the FP32 residual has dropped by `delta` since the last
// replacement (or below the final threshold), the FP32 increment is folded into the FP64 iterate
// x, the true residual b - K x is formed in FP64 with the matrix-free tangent (the operator the
// FP64 path assembles), and the FP32 residual is replaced by it; the search direction is kept,
// so the Krylov space is not thrown away as a restarted defect correction does.  Stops when
// the true residual meets ||r|| < tol ||b|| (the PCG's stop test, linear_solver.cpp:67-109).
int pcg_reliable_mixed(nb2_ctx* c, const double* b, double* x, double tol, double delta,
                       int maxit, double* work, int* iterations, bool use_graphs,
                       bool matrix_free) {
    CgRunner<float, float> cg{c,         c->K32,      c->cg32_x, c->cg32_r, c->cg32_p,
                              c->cg32_q, c->cg32_inv, true,      use_graphs,
                              matrix_free ? &c->graph_mf : &c->graph32};
    cg.mf = matrix_free;
    if (matrix_free) {
        // FP32 operator data and the Jacobi inverse from the stored tangent
        NB2_TRY(ensure_mf(c));
        NB2_TRY(launch_mf_setup(c));
        k_mf_diag<<<(c->N + 255) / 256, 256, 0, c->stream>>>(c->N, c->nadj_ptr, c->nadj_pl,
                                                             c->mf_ye, c->cg32_inv);
        c->launches++;
    }
    NB2_TRY(cg.setup());
    const long long n = c->n;
    const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, 148 * 8);
    NB2_CUDA(c, cudaMemsetAsync(x, 0, sizeof(double) * n, c->stream));
    // the first pause comes after a delta reduction of ||b|| (threshold max(tol, delta)^2 b.b)
    const double t0 = std::max(tol, delta);
    k_init<float><<<cg.RB, kRedThreads, 0, c->stream>>>(n, b, cg.x, cg.r, cg.p, cg.inv, c->cgs,
                                                        c->partials, t0);
    c->launches++;
    NB2_CUDA(c, cudaMemcpyAsync(&c->cgs->max_iterations, &maxit, sizeof(int),
                                cudaMemcpyHostToDevice, c->stream));
    NB2_TRY(wait_scalars(c));
    const double b2 = c->h_cgs->rhs_norm2;
    const double thr = std::max(tol * tol * b2, 2.2250738585072014e-308);
    *iterations = 0;
    if (b2 == 0.0) return NB2_OK;
    double* rr_dev = c->norms + 6;
    int resets = 0;
    for (int update = 0;; ++update) {
        if (!c->h_cgs->done) NB2_TRY(cg.run(maxit));
        const CgScalars h = *c->h_cgs;
        *iterations = h.iterations;
        // a diverged cycle (its kept search direction no longer fits the replaced residual,
        // near the FP32 operator's accuracy floor): replace the residual again and restart the
        // cycle with p = D^-1 r, at most three times per solve
        const bool fresh = h.status == NB2_E_CG_BREAKDOWN && resets < 3;
        if (fresh) ++resets;
        if (h.status && h.status != NB2_E_CG_MAXIT && !fresh) return h.status;
        // reliable update: x += xs; r = b - K x in FP64
        k_fold<<<grid, 256, 0, c->stream>>>(n, cg.x, x);
        NB2_TRY(launch_apply(c, x, work));
        k_true_residual<<<cg.RB, kRedThreads, 0, c->stream>>>(n, b, work, c->mask, cg.inv, cg.r,
                                                              c->cgs, c->partials, rr_dev);
        c->launches += 2;
        double rr = 0;
        NB2_CUDA(c, cudaMemcpyAsync(&rr, rr_dev, sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream));
        NB2_CUDA(c, cudaStreamSynchronize(c->stream));
        if (std::getenv("NB2_DEBUG"))
            std::fprintf(stderr, "[nb2] reliable update %d: its %d true |r|^2 %.6e thr %.6e\n",
                         update, h.iterations, rr, thr);
        if (!std::isfinite(rr)) return NB2_E_NAN;
        if (rr < thr) return NB2_OK;
        if (h.status == NB2_E_CG_MAXIT || h.iterations >= maxit || update > 1000)
            return NB2_E_CG_MAXIT;
        // continue: p = D^-1 r + beta p with the replaced residual, next pause after delta
        const double next = std::max(thr, delta * delta * rr);
        CgScalars upd = h;
        upd.threshold = next;
        upd.done = 0;
        upd.status = 0;
        NB2_CUDA(c, cudaMemcpyAsync(&c->cgs->threshold, &upd.threshold, sizeof(double),
                                    cudaMemcpyHostToDevice, c->stream));
        NB2_CUDA(c, cudaMemcpyAsync(&c->cgs->done, &upd.done, sizeof(int), cudaMemcpyHostToDevice,
                                    c->stream));
        NB2_CUDA(c, cudaMemcpyAsync(&c->cgs->status, &upd.status, sizeof(int),
                                    cudaMemcpyHostToDevice, c->stream));
        if (fresh) {
            static const double zero = 0.0;
            NB2_CUDA(c, cudaMemcpyAsync(&c->cgs->beta, &zero, sizeof(double),
                                        cudaMemcpyHostToDevice, c->stream));
        }
        k_p<float><<<cg.RB, kRedThreads, 0, c->stream>>>(n, cg.p, cg.r, cg.inv, c->cgs);
        c->launches++;
        NB2_TRY(wait_scalars(c));
    }
}

int pcg_device_fp64(nb2_ctx* c, const double* b, double* x, double tol, int maxit, bool use_mask,
                    int* iterations, double* error, bool use_graphs) {
    return run_bsr_cg<double, double>(c, c->K64, c->cg_x, c->cg_r, c->cg_p, c->cg_q, c->cg_inv, b,
                                      x, tol, maxit, use_mask, iterations, error,
                                      use_graphs && use_mask, &c->graph64[c->kbuf]);
}

int pcg_device_fp32(nb2_ctx* c, const double* b, double* x, double tol, int maxit, int* iterations,
                    double* error, bool use_graphs) {
    return run_bsr_cg<float, float>(c, c->K32, c->cg32_x, c->cg32_r, c->cg32_p, c->cg32_q,
                                    c->cg32_inv, b, x, tol, maxit, true, iterations, error,
                                    use_graphs, &c->graph32);
}

void release_graphs(nb2_ctx* c) {
    for (auto& g : c->graph64) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    if (c->graph32) cudaGraphExecDestroy(c->graph32);
    if (c->graph_mf) cudaGraphExecDestroy(c->graph_mf);
    c->graph32 = c->graph_mf = nullptr;
}

// y = K v with the FP32 matrix-free operator (v, y device FP64; y unmasked)
int mf_apply(nb2_ctx* c, const double* v, double* y) {
    NB2_TRY(ensure_k32(c));
    NB2_TRY(ensure_mf(c));
    NB2_TRY(launch_mf_setup(c));
    const long long n = c->n;
    k_to_float<<<(unsigned)std::min<long long>((n + 255) / 256, 148 * 8), 256, 0, c->stream>>>(
        n, v, c->cg32_p);
    enqueue_apply32(c, c->cg32_p, c->mf_ye, nullptr);
    k_mf_sum<<<(c->N + 255) / 256, 256, 0, c->stream>>>(c->N, c->nadj_ptr, c->nadj_pl, c->mf_ye, y);
    c->launches += 3;
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

// slot e*npe + a of the node adjacency -> its position a*E + e in the per-node planes of mf_ye
__global__ void k_plane_slots(long long m, int npe, int E, const int* __restrict__ nadj,
                              int* __restrict__ nadj_pl) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int sl = nadj[k];
    nadj_pl[k] = (sl % npe) * E + sl / npe;
}

int ensure_mf(nb2_ctx* c) {
    if (c->mf_d) return NB2_OK;
    const long long ev = (long long)c->E * c->npe * 3;
    NB2_CUDA(c, cudaMalloc(&c->mf_d, sizeof(float) * ev));
    NB2_CUDA(c, cudaMalloc(&c->mf_ye, sizeof(float) * ev));
    NB2_CUDA(c, cudaMalloc(&c->mf_c, sizeof(float) * (long long)mf_coefficients(c->mat.model) *
                                         c->nqp));
    NB2_TRY(build_node_adjacency(c));
    const long long m = (long long)c->E * c->npe;
    NB2_CUDA(c, cudaMalloc(&c->nadj_pl, sizeof(int) * m));
    k_plane_slots<<<(unsigned)((m + 255) / 256), 256, 0, c->stream>>>(m, c->npe, c->E, c->nadj,
                                                                       c->nadj_pl);
    c->launches++;
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

void bsr_spmv_fp64(nb2_ctx* c, const double* x, double* y, bool use_mask) {
    Bsr<double> A{c->brp, c->bcol, c->K64, c->N};
    k_bsr_apply<double><<<reduction_blocks(c), kRedThreads, 0, c->stream>>>(
        A, x, y, use_mask ? c->mask : nullptr);
    c->launches++;
}

void bsr_spmv_mixed_accum(nb2_ctx* c, const double* x, double* y) {
    Bsr<float> A{c->brp, c->bcol, c->K32, c->N};
    k_bsr_apply<float><<<reduction_blocks(c), kRedThreads, 0, c->stream>>>(A, x, y, nullptr);
    c->launches++;
}

__global__ void __launch_bounds__(kRedThreads) k_dot1(long long n, const double* a, const double* b,
                                                      double* partials, unsigned int* counter,
                                                      double* out) {
    double acc[1] = {0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        acc[0] += a[i] * b[i];
    if (block_partials<1>(acc, partials, counter)) {
        double tot[1];
        final_sum<1>(partials, tot);
        if (threadIdx.x == 0) {
            *out = tot[0];
            *counter = 0;
        }
    }
}

double device_dot_sync(nb2_ctx* c, const double* a, const double* b, int n) {
    k_dot1<<<reduction_blocks(c), kRedThreads, 0, c->stream>>>(n, a, b, c->partials,
                                                                &c->cgs->counter[3], c->norms + 5);
    c->launches++;
    cudaMemcpyAsync(c->h_norms + 5, c->norms + 5, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    cudaStreamSynchronize(c->stream);
    return c->h_norms[5];
}

int compute_norms(nb2_ctx* c) {
    k_norms<<<reduction_blocks(c), kRedThreads, 0, c->stream>>>(
        c->n, c->du, c->u, c->rhs, c->fext, c->fint, c->partials, &c->cgs->counter[3], c->norms);
    c->launches++;
    NB2_CUDA(c, cudaMemcpyAsync(c->h_norms, c->norms, 5 * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

// Standalone solve on a caller CSR (host buffers): own stream and buffers.
int pcg_csr_host(int n, const int* rowptr, const int* col, const double* val, const double* b,
                 double* x, double tol, int maxit, int* iterations, double* error,
                 std::string* err) {
    nb2_ctx tmp;
    nb2_ctx* c = &tmp;
    auto fail = [&](cudaError_t e) {
        if (err) *err = cudaGetErrorString(e);
        return NB2_E_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(e);
    const long long nnz = rowptr[n];
    int *rp = nullptr, *ci = nullptr;
    double *v = nullptr, *bd = nullptr, *xd = nullptr, *r = nullptr, *p = nullptr, *q = nullptr,
           *inv = nullptr, *xo = nullptr, *partials = nullptr;
    CgScalars* s = nullptr;
    CgScalars hs;
    const int RB = 148 * 4;
    int status = NB2_OK;
#define TRY(call)                          \
    if ((e = (call)) != cudaSuccess) {     \
        status = fail(e);                  \
        goto done;                         \
    }
    TRY(cudaMalloc(&rp, sizeof(int) * (n + 1)));
    TRY(cudaMalloc(&ci, sizeof(int) * (nnz > 0 ? nnz : 1)));
    TRY(cudaMalloc(&v, sizeof(double) * (nnz > 0 ? nnz : 1)));
    TRY(cudaMalloc(&bd, sizeof(double) * n));
    TRY(cudaMalloc(&xd, sizeof(double) * n));
    TRY(cudaMalloc(&r, sizeof(double) * n));
    TRY(cudaMalloc(&p, sizeof(double) * n));
    TRY(cudaMalloc(&q, sizeof(double) * n));
    TRY(cudaMalloc(&inv, sizeof(double) * n));
    TRY(cudaMalloc(&xo, sizeof(double) * n));
    TRY(cudaMalloc(&partials, sizeof(double) * RB * 8));
    TRY(cudaMalloc(&s, sizeof(CgScalars)));
    TRY(cudaMemsetAsync(s, 0, sizeof(CgScalars), c->stream));
    TRY(cudaMemcpyAsync(rp, rowptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, c->stream));
    TRY(cudaMemcpyAsync(ci, col, sizeof(int) * nnz, cudaMemcpyHostToDevice, c->stream));
    TRY(cudaMemcpyAsync(v, val, sizeof(double) * nnz, cudaMemcpyHostToDevice, c->stream));
    TRY(cudaMemcpyAsync(bd, b, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    TRY(cudaMemcpyAsync(&s->max_iterations, &maxit, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    {
        Csr A{rp, ci, v, n};
        k_csr_invdiag<<<(n + 255) / 256, 256, 0, c->stream>>>(A, inv);
        k_init<double><<<RB, kRedThreads, 0, c->stream>>>(n, bd, xd, r, p, inv, s, partials, tol);
        TRY(cudaMemcpyAsync(&s->max_iterations, &maxit, sizeof(int), cudaMemcpyHostToDevice,
                            c->stream));
        int guard = 0;
        for (;;) {
            if (++guard > maxit / kChunk + 4) {
                status = NB2_E_TIMEOUT;
                goto done;
            }
            for (int it = 0; it < kChunk; ++it) {
                k_csr_spmv<<<RB, kRedThreads, 0, c->stream>>>(A, p, q, s, partials);
                k_xr<double><<<RB, kRedThreads, 0, c->stream>>>(n, xd, r, p, q, inv, s, partials);
                k_p<double><<<RB, kRedThreads, 0, c->stream>>>(n, p, r, inv, s);
            }
            TRY(cudaMemcpyAsync(&hs, s, sizeof hs, cudaMemcpyDeviceToHost, c->stream));
            TRY(cudaStreamSynchronize(c->stream));
            if (hs.done) break;
        }
        TRY(cudaGetLastError());
        TRY(cudaMemcpyAsync(x, xd, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
        TRY(cudaStreamSynchronize(c->stream));
        *iterations = hs.iterations;
        *error = hs.rhs_norm2 > 0 ? std::sqrt(hs.rr / hs.rhs_norm2) : 0.0;
        if (hs.status) status = hs.status;
    }
done:
#undef TRY
    cudaFree(rp);
    cudaFree(ci);
    cudaFree(v);
    cudaFree(bd);
    cudaFree(xd);
    cudaFree(r);
    cudaFree(p);
    cudaFree(q);
    cudaFree(inv);
    cudaFree(xo);
    cudaFree(partials);
    cudaFree(s);
    cudaStreamDestroy(c->stream);
    c->stream = nullptr;
    return status;
}

// ---------------------------------------------------------------------------------------
// Allocation-free PCG (nb2_pcg_solve_noalloc).
//
// For callers that must not allocate device memory while they run a solve: a code that places
// every device byte itself through its own pool or arena and forbids hidden allocations, or a
// long-running service that must not trigger allocator growth in the middle of a time step.
// They pass the matrix, right-hand side and solution in device memory they own; the solver's
// own work vectors, reduction partials and scalars live in the fixed array below, which every
// GPU that loads this library holds until the process exits.  The call allocates nothing, but
// it is not asynchronous: it blocks the host on its stream after the CSR check and once every
// kChunk iterations to read the convergence flag, so it cannot run inside a stream capture.
// ---------------------------------------------------------------------------------------
constexpr int kNoAllocMaxRows = NB2_NOALLOC_MAX_ROWS;
constexpr int kNoAllocBlocks = 148 * 4;
// layout (doubles): [partials kNoAllocBlocks*8][scalars 32][r][p][q][inv] (rows each)
constexpr size_t kNoAllocPartials = (size_t)kNoAllocBlocks * 8;
constexpr size_t kNoAllocScalars = 32;  // >= sizeof(CgScalars) / 8, keeps 256-byte alignment
constexpr size_t kNoAllocDoubles = kNoAllocPartials + kNoAllocScalars + 4ull * kNoAllocMaxRows;
static_assert(sizeof(CgScalars) <= kNoAllocScalars * sizeof(double), "scalar slot too small");

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// row pointers monotone from 0; flag = 1 on any violation.  Run first, and its flag read back,
// so that the column check below never walks past a corrupt rp[n]
__global__ void k_check_rowptr(int n, const int* __restrict__ rp, unsigned int* flag) {
    const int nnz = rp[n];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (rp[i + 1] < rp[i] || rp[i] < 0 || rp[i + 1] > nnz) atomicOr(flag, 1u);
    if (blockIdx.x == 0 && threadIdx.x == 0 && (rp[0] != 0 || nnz < 0)) atomicOr(flag, 1u);
}

// column indices in [0, n) over [0, rp[n]) (rp already checked); flag = 1 on any violation
__global__ void k_check_columns(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                unsigned int* flag) {
    const long long nnz = rp[n];
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x)
        if (ci[k] < 0 || ci[k] >= n) atomicOr(flag, 1u);
}

}  // namespace nb2

extern "C" int nb2_pcg_solve_noalloc(int32_t n, const int32_t* rowptr, const int32_t* col,
                                     const double* values, const double* b, double* x,
                                     double tolerance, int32_t maximum_iterations, void* stream,
                                     int32_t* iterations, double* error) {
    using namespace nb2;
    if (n <= 0 || !rowptr || !col || !values || !b || !x || maximum_iterations <= 0)
        return NB2_E_INPUT;
    if (n > kNoAllocMaxRows) return NB2_E_INPUT;  // beyond the fixed workspace
    // device address of the fixed workspace, looked up on every call with the caller's device
    // current (the symbol's host-side name is not a device address).  The lookup allocates
    // nothing; doing it per call keeps no pointer that a cudaDeviceReset could leave stale.
    // The first call on a device loads the library's module there, so make it before any
    // stream capture.
    void* sym = nullptr;
    if (cudaGetSymbolAddress(&sym, g_noalloc_scratch) != cudaSuccess || !sym) return NB2_E_CUDA;
    double* base = static_cast<double*>(sym);
    double* partials = base;
    CgScalars* s = reinterpret_cast<CgScalars*>(base + kNoAllocPartials);
    double* r = base + kNoAllocPartials + kNoAllocScalars;
    double* p = r + kNoAllocMaxRows;
    double* q = p + kNoAllocMaxRows;
    double* inv = q + kNoAllocMaxRows;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int RB = kNoAllocBlocks;
    // the workspace keeps the previous call's contents: the scalars (reduction tickets, flags)
    // must start at zero
    if (cudaMemsetAsync(s, 0, sizeof(CgScalars), st) != cudaSuccess) return NB2_E_CUDA;
    unsigned int* flag = &s->counter[3];
    CgScalars hs;
    auto read_flag = [&](unsigned int* out) {
        if (cudaMemcpyAsync(&hs, s, sizeof hs, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return false;
        *out = hs.counter[3];
        return true;
    };
    unsigned int bad = 0;
    k_check_rowptr<<<RB, kRedThreads, 0, st>>>(n, rowptr, flag);
    if (!read_flag(&bad)) return NB2_E_CUDA;
    if (bad != 0) return NB2_E_INPUT;
    k_check_columns<<<RB, kRedThreads, 0, st>>>(n, rowptr, col, flag);
    if (!read_flag(&bad)) return NB2_E_CUDA;
    if (bad != 0) return NB2_E_INPUT;
    if (cudaMemsetAsync(s, 0, sizeof(CgScalars), st) != cudaSuccess) return NB2_E_CUDA;
    if (cudaMemcpyAsync(&s->max_iterations, &maximum_iterations, sizeof(int),
                        cudaMemcpyHostToDevice, st) != cudaSuccess)
        return NB2_E_CUDA;
    Csr A{rowptr, col, values, n};
    k_csr_invdiag<<<(n + 255) / 256, 256, 0, st>>>(A, inv);
    k_init<double><<<RB, kRedThreads, 0, st>>>(n, b, x, r, p, inv, s, partials, tolerance);
    int guard = 0;
    for (;;) {
        if (++guard > maximum_iterations / kChunk + 4) return NB2_E_TIMEOUT;
        for (int it = 0; it < kChunk; ++it) {
            k_csr_spmv<<<RB, kRedThreads, 0, st>>>(A, p, q, s, partials);
            k_xr<double><<<RB, kRedThreads, 0, st>>>(n, x, r, p, q, inv, s, partials);
            k_p<double><<<RB, kRedThreads, 0, st>>>(n, p, r, inv, s);
        }
        if (cudaMemcpyAsync(&hs, s, sizeof hs, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return NB2_E_CUDA;
        if (hs.done) break;
    }
    if (cudaGetLastError() != cudaSuccess) return NB2_E_CUDA;
    if (iterations) *iterations = hs.iterations;
    if (error) *error = hs.rhs_norm2 > 0 ? std::sqrt(hs.rr / hs.rhs_norm2) : 0.0;
    return hs.status ? hs.status : NB2_OK;
}
