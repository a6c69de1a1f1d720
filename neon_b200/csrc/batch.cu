// batch.cu -- many independent problems (instances) of uneven size in one context.
//
// The instances are stored as one block-diagonal mesh (instance i owns a contiguous node range
// and the elements on it; per-element moduli carry each instance's material), so every element
// pass, SpMV and vector update covers all instances in a single launch.  What neon keeps per
// problem stays per instance: the load stepping (adaptive_time_step.cpp:12-165), the Newton
// decisions and norms (static_matrix.hpp:145-187, 353-467) and the PCG scalars
// (linear_solver.cpp:67-109).  Rows are cut into chunks that never straddle two instances; each
// PCG kernel takes one chunk per CTA, writes a per-chunk partial, and the last chunk of an
// instance to finish (a per-instance ticket) reduces that instance's partials in a fixed order:
// deterministic segmented reductions with no spin waits.  An instance that has converged (or is
// between load increments) is skipped by every kernel.  The rows per chunk and the lanes per
// block row of the SpMV are chosen by timing (nb2_batch_autotune).
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host_driver.hpp"
#include "nb2_internal.cuh"

namespace nb2 {

namespace {

constexpr int kThreads = 256;
constexpr int kBatchChunk = 32;  // CG iterations per captured graph
// operator / vector precision of the batched PCG
constexpr int kModeK64 = 0;    // FP64 K, FP64 vectors
constexpr int kModeK32V64 = 1; // FP32 K, FP64 vectors (the batched mixed path)

// a cycle of the mixed reliable-update PCG whose FP32 recurrence residual has grown to this
// multiple of its squared norm at the residual replacement has diverged (CG residual norms are
// not monotone, so the margin is wide: a factor 1000 in the norm)
constexpr double kCycleDivergence = 1e6;

struct Tables {
    const int* row0;   // [nchunks] first block row
    const int* row1;   // [nchunks] one past the last
    const int* inst;   // [nchunks] owning instance
    const int* first;  // [ninst] first chunk of the instance
    const int* count;  // [ninst] chunks of the instance
};

// per-instance PCG scalars, structure of arrays of length ninst
struct Scalars {
    double *rhs2, *thr, *absnew, *pq, *alpha, *rr, *beta;
    double* rrcap;     // recurrence residual above which a reliable-update cycle has diverged
    int *iters, *done, *status, *maxit;
    unsigned* ticket;  // [4][ninst]
    int ninst;
    int timing;        // autotuner sweeps: leave the scalars alone
};

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// CTA sums of NV values into part[blk * NV + j]; true in the CTA that completes the instance
template <int NV>
__device__ bool chunk_partials(double (&v)[NV], double* part, unsigned* ticket, int count) {
    __shared__ double red[NV][kThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const double t = wsum(v[j]);
        if (lane == 0) red[j][wid] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double t = 0;
            for (int w = 0; w < kThreads / 32; ++w) t += red[j][w];
            part[blockIdx.x * NV + j] = t;
        }
        __threadfence();
        last = atomicAdd(ticket, 1u) == (unsigned)count - 1;
    }
    __syncthreads();
    return last;
}

// fixed-order sum of the instance's chunk partials (whole CTA)
template <int NV>
__device__ void instance_sum(const double* part, int first, int count, double (&out)[NV]) {
    __shared__ double red[NV][kThreads];
    __threadfence();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double t = 0;
        for (int b = threadIdx.x; b < count; b += kThreads)
            t += *((volatile const double*)&part[(long long)(first + b) * NV + j]);
        red[j][threadIdx.x] = t;
    }
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
#pragma unroll
            for (int j = 0; j < NV; ++j) red[j][threadIdx.x] += red[j][threadIdx.x + s];
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < NV; ++j) out[j] = red[j][0];
}

template <typename X>
__global__ void __launch_bounds__(kThreads) k_b_init(Tables T, const double* __restrict__ b,
                                                     X* x, X* r, X* p, const X* inv, Scalars S,
                                                     double* part, double tol) {
    const int inst = T.inst[blockIdx.x];
    const long long i0 = 3ll * T.row0[blockIdx.x], i1 = 3ll * T.row1[blockIdx.x];
    double acc[3] = {0, 0, 0};
    for (long long i = i0 + threadIdx.x; i < i1; i += kThreads) {
        const X bi = (X)b[i];
        x[i] = (X)0;
        r[i] = bi;
        const X pi = inv[i] * bi;
        p[i] = pi;
        acc[0] += b[i] * b[i];
        acc[1] += (double)bi * (double)bi;
        acc[2] += (double)bi * (double)pi;
    }
    if (chunk_partials<3>(acc, part, &S.ticket[2 * S.ninst + inst], T.count[inst])) {
        double tot[3];
        instance_sum<3>(part, T.first[inst], T.count[inst], tot);
        if (threadIdx.x == 0) {
            S.rhs2[inst] = tot[0];
            S.thr[inst] = fmax(tol * tol * tot[0], DBL_MIN);
            S.rr[inst] = tot[1];
            S.rrcap[inst] = INFINITY;
            S.absnew[inst] = tot[2];
            S.iters[inst] = 0;
            S.status[inst] = 0;
            S.done[inst] = (tot[0] == 0.0 || tot[1] < S.thr[inst]) ? 1 : 0;
            S.ticket[2 * S.ninst + inst] = 0;
        }
    }
}

// q = K p (masked rows 0) with LPR lanes per block row, and the instance's p.q -> alpha
template <typename V, typename X, int LPR>
__global__ void __launch_bounds__(kThreads) k_b_spmv(Tables T, const int* __restrict__ brp,
                                                     const int* __restrict__ bcol,
                                                     const V* __restrict__ val,
                                                     const X* __restrict__ p, X* __restrict__ q,
                                                     const unsigned char* __restrict__ mask,
                                                     Scalars S, double* part,
                                                     const float* __restrict__ dc) {
    const int inst = T.inst[blockIdx.x];
    if (S.done[inst]) return;
    constexpr int RPW = 32 / LPR;  // rows of a warp in flight
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sub = lane / LPR, sl = lane % LPR;
    const int r0 = T.row0[blockIdx.x], r1 = T.row1[blockIdx.x];
    double dot[1] = {0.0};
    for (int a0 = r0 + warp * RPW; a0 < r1; a0 += (kThreads / 32) * RPW) {
        const int a = a0 + sub;
        X y0 = 0, y1 = 0, y2 = 0;
        if (a < r1) {
            const int b0 = brp[a], b1 = brp[a + 1];
            for (int k = b0 + sl; k < b1; k += LPR) {
                const long long col = bcol[k];
                const X x0 = p[3 * col], x1 = p[3 * col + 1], x2 = p[3 * col + 2];
                const V* blk = val + 9ll * k;
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
        if (a < r1 && sl < 3) {
            const long long i = 3ll * a + sl;
            X y = sl == 0 ? y0 : (sl == 1 ? y1 : y2);
            if (dc) y += (X)dc[i] * p[i];
            if (mask && mask[i]) y = (X)0;
            q[i] = y;
            dot[0] += (double)p[i] * (double)y;
        }
    }
    if (chunk_partials<1>(dot, part, &S.ticket[inst], T.count[inst])) {
        double tot[1];
        instance_sum<1>(part, T.first[inst], T.count[inst], tot);
        if (threadIdx.x == 0) {
            if (!S.timing) {
                S.pq[inst] = tot[0];
                S.alpha[inst] = S.absnew[inst] / tot[0];
                if (!isfinite(S.alpha[inst])) {
                    S.status[inst] = NB2_E_NAN;
                    S.done[inst] = 1;
                }
            }
            S.ticket[inst] = 0;
        }
    }
}

template <typename X>
__global__ void __launch_bounds__(kThreads) k_b_xr(Tables T, X* x, X* r, const X* p, const X* q,
                                                   const X* inv, Scalars S, double* part) {
    const int inst = T.inst[blockIdx.x];
    if (S.done[inst]) return;
    const X alpha = (X)S.alpha[inst];
    const long long i0 = 3ll * T.row0[blockIdx.x], i1 = 3ll * T.row1[blockIdx.x];
    double acc[2] = {0.0, 0.0};
    for (long long i = i0 + threadIdx.x; i < i1; i += kThreads) {
        x[i] += alpha * p[i];
        const X ri = r[i] - alpha * q[i];
        r[i] = ri;
        acc[0] += (double)ri * (double)ri;
        acc[1] += (double)ri * (double)(inv[i] * ri);
    }
    if (chunk_partials<2>(acc, part, &S.ticket[S.ninst + inst], T.count[inst])) {
        double tot[2];
        instance_sum<2>(part, T.first[inst], T.count[inst], tot);
        if (threadIdx.x == 0) {
            S.rr[inst] = tot[0];
            if (!isfinite(tot[0])) {
                S.done[inst] = 1;
                S.status[inst] = NB2_E_NAN;
            } else if (tot[0] < S.thr[inst]) {
                S.done[inst] = 1;
            } else if (tot[0] > S.rrcap[inst]) {
                S.done[inst] = 1;
                S.status[inst] = NB2_E_CG_BREAKDOWN;
            } else {
                S.beta[inst] = tot[1] / S.absnew[inst];
                S.absnew[inst] = tot[1];
                if (++S.iters[inst] >= S.maxit[inst]) {
                    S.done[inst] = 1;
                    S.status[inst] = NB2_E_CG_MAXIT;
                }
            }
            S.ticket[S.ninst + inst] = 0;
        }
    }
}

template <typename X>
__global__ void __launch_bounds__(kThreads) k_b_p(Tables T, X* p, const X* r, const X* inv,
                                                  Scalars S) {
    const int inst = T.inst[blockIdx.x];
    if (S.done[inst]) return;
    const X beta = (X)S.beta[inst];
    const long long i0 = 3ll * T.row0[blockIdx.x], i1 = 3ll * T.row1[blockIdx.x];
    for (long long i = i0 + threadIdx.x; i < i1; i += kThreads) p[i] = inv[i] * r[i] + beta * p[i];
}

// per-instance 2-norms of up to 5 vectors (null entries give 0): out[k * ninst + inst]
__global__ void __launch_bounds__(kThreads) k_b_norms(Tables T, const double* v0, const double* v1,
                                                      const double* v2, const double* v3,
                                                      const double* v4, Scalars S, double* part,
                                                      double* out) {
    const int inst = T.inst[blockIdx.x];
    const long long i0 = 3ll * T.row0[blockIdx.x], i1 = 3ll * T.row1[blockIdx.x];
    const double* v[5] = {v0, v1, v2, v3, v4};
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long i = i0 + threadIdx.x; i < i1; i += kThreads)
#pragma unroll
        for (int k = 0; k < 5; ++k)
            if (v[k]) acc[k] += v[k][i] * v[k][i];
    if (chunk_partials<5>(acc, part, &S.ticket[3 * S.ninst + inst], T.count[inst])) {
        double tot[5];
        instance_sum<5>(part, T.first[inst], T.count[inst], tot);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < 5; ++k) out[k * S.ninst + inst] = sqrt(tot[k]);
            S.ticket[3 * S.ninst + inst] = 0;
        }
    }
}

// v[rows of instance i] = value where (flag[i] != 0) == want
template <typename T>
__global__ void k_b_fill(Tables Tb, const int* flag, int want, T* v, T value) {
    const int inst = Tb.inst[blockIdx.x];
    if ((flag[inst] != 0) != (want != 0)) return;
    const long long i0 = 3ll * Tb.row0[blockIdx.x], i1 = 3ll * Tb.row1[blockIdx.x];
    for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) v[i] = value;
}

// dst[rows of instance i] = src where flag[i] != 0
__global__ void k_b_copy(Tables Tb, const int* flag, const double* src, double* dst) {
    const int inst = Tb.inst[blockIdx.x];
    if (!flag[inst]) return;
    const long long i0 = 3ll * Tb.row0[blockIdx.x], i1 = 3ll * Tb.row1[blockIdx.x];
    for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) dst[i] = src[i];
}

__global__ void k_b_sub(long long n, const double* a, const double* b, double* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = a[i] - b[i];
}

__global__ void k_b_axpy(long long n, double alpha, const double* x, double* y) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] += alpha * x[i];
}

__global__ void k_b_zero_masked(long long n, const unsigned char* mask, double* v) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (mask[i]) v[i] = 0.0;
}

// Dirichlet entries of the tables switched on this round: mask the DOF, set its increment
__global__ void k_b_dirichlet(int m, const int* dofs, const int* tab, const int* on,
                              const double* delta, unsigned char* mask, double* inc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int t = tab[i];
    if (!on[t]) return;
    mask[dofs[i]] = 1;
    inc[dofs[i]] = delta[t];
}

// nodal-force entries of the tables switched on this round: f_ext[dof] += w value(t)
__global__ void k_b_forces(int m, const int* dofs, const int* tab, const double* w,
                           const int* on, const double* value, double* fext) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int t = tab[i];
    if (!on[t]) return;
    atomicAdd(&fext[dofs[i]], (w ? w[i] : 1.0) * value[t]);
}

// element -> instance by its first node; bad[0] counts elements that couple two instances
__global__ void k_b_element_instance(long long E, int npe, const int* conn, const int* offsets,
                                     int ninst, int* e_inst, int* bad) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int n0 = conn[e * npe];
    int lo = 0, hi = ninst - 1;  // last instance with offsets[i] <= n0
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (offsets[mid] <= n0) lo = mid; else hi = mid - 1;
    }
    e_inst[e] = lo;
    for (int a = 1; a < npe; ++a) {
        const int nd = conn[e * npe + a];
        if (nd < offsets[lo] || nd >= offsets[lo + 1]) {
            atomicAdd(bad, 1);
            break;
        }
    }
}

template <typename V, typename X>
__global__ void k_b_invdiag(const int* brp, const int* bcol, const V* val, int rows, X* inv) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= rows) return;
    int lo = brp[a], hi = brp[a + 1] - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (bcol[mid] < a) lo = mid + 1; else hi = mid;
    }
    const bool has = lo < brp[a + 1] && bcol[lo] == a;  // empty row: diagonal 0
    for (int r = 0; r < 3; ++r) {
        const double d = has ? (double)val[9ll * lo + 4 * r] : 0.0;
        inv[3ll * a + r] = d != 0.0 ? (X)(1.0 / d) : (X)1;
    }
}

// FP32 K with a compensated diagonal.  The tangent of any of these models is unchanged by a
// rigid translation (f_int does not move when every node does), so in each row the entries of
// one component sum to zero: K_(3a+r, 3a+r) = -sum_(b != a) K_(3a+r, 3b+r).  Rounding K to FP32
// breaks that identity by about the rounding of the diagonal, which is the largest entry, and
// the translation-like modes that give the small eigenvalues then see a relatively large
// operator error.  dc restores it: dc = -(sum of the FP32 off-diagonal same-component entries,
// in FP64) - (FP32 diagonal), added as dc p in the SpMV, so the operator's diagonal is the
// compensated value and every row sums to zero again to FP64 rounding.  The Jacobi inverse uses
// the same diagonal (1 where it is 0).
__global__ void k_b_compdiag(const int* brp, const int* bcol, const float* val, int rows,
                             float* dc, double* inv) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= rows) return;
    double off[3] = {0.0, 0.0, 0.0}, d[3] = {0.0, 0.0, 0.0};
    for (int k = brp[a]; k < brp[a + 1]; ++k) {
        const float* blk = val + 9ll * k;
        if (bcol[k] == a) {
            for (int r = 0; r < 3; ++r) d[r] = (double)blk[4 * r];
        } else {
            for (int r = 0; r < 3; ++r) off[r] += (double)blk[4 * r];
        }
    }
    for (int r = 0; r < 3; ++r) {
        const double dd = -off[r];
        dc[3ll * a + r] = (float)(dd - d[r]);
        inv[3ll * a + r] = dd != 0.0 ? 1.0 / dd : 1.0;
    }
}

template <typename X>
__global__ void k_b_out(long long n, const X* x, double* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (double)x[i];
}

// Residual replacement of the flagged instances: r = b - y (FP64, masked rows 0), rs = (X)r;
// per instance r.r -> rr_out[inst] and the recurrence continued with rz_new = rs.D^-1 rs
template <typename X>
__global__ void __launch_bounds__(kThreads) k_b_true_residual(Tables T, const int* flag,
                                                              const double* __restrict__ b,
                                                              const double* __restrict__ y,
                                                              const unsigned char* __restrict__ mask,
                                                              const X* __restrict__ inv,
                                                              X* __restrict__ rs, Scalars S,
                                                              double* part, double* rr_out) {
    const int inst = T.inst[blockIdx.x];
    if (!flag[inst]) return;
    const long long i0 = 3ll * T.row0[blockIdx.x], i1 = 3ll * T.row1[blockIdx.x];
    double acc[2] = {0.0, 0.0};
    for (long long i = i0 + threadIdx.x; i < i1; i += kThreads) {
        const double ri = mask[i] ? 0.0 : b[i] - y[i];
        const X rf = (X)ri;
        rs[i] = rf;
        acc[0] += ri * ri;
        acc[1] += (double)rf * (double)(inv[i] * rf);
    }
    if (chunk_partials<2>(acc, part, &S.ticket[3 * S.ninst + inst], T.count[inst])) {
        double tot[2];
        instance_sum<2>(part, T.first[inst], T.count[inst], tot);
        if (threadIdx.x == 0) {
            rr_out[inst] = tot[0];
            S.rr[inst] = tot[0];
            S.rrcap[inst] = kCycleDivergence * tot[0];
            S.beta[inst] = tot[1] / S.absnew[inst];
            S.absnew[inst] = tot[1];
            S.ticket[3 * S.ninst + inst] = 0;
        }
    }
}

// restart the flagged instances' cycle from the replaced residual with a fresh search
// direction (beta = 0) and a cleared status
__global__ void k_b_restart_cycle(int ninst, const int* flag, Scalars S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst || !flag[i]) return;
    S.beta[i] = 0.0;
    S.status[i] = NB2_OK;
}

unsigned vgrid(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148 * 8); }

template <typename V, typename X>
using SpmvFn = void (*)(Tables, const int*, const int*, const V*, const X*, X*,
                        const unsigned char*, Scalars, double*, const float*);

template <typename V, typename X>
SpmvFn<V, X> spmv_variant(int lanes) {
    switch (lanes) {
        case 4: return k_b_spmv<V, X, 4>;
        case 8: return k_b_spmv<V, X, 8>;
        case 16: return k_b_spmv<V, X, 16>;
        default: return k_b_spmv<V, X, 32>;
    }
}

// ---------------------------------------------------------------------------------------
// host side: chunk tables and per-instance scalars
// ---------------------------------------------------------------------------------------
struct BatchState {
    int ninst = 0, nchunks = 0, rows = 32, lanes = 16;
    std::vector<int> h_first, h_count, h_node_off;
    int *row0 = nullptr, *row1 = nullptr, *inst = nullptr, *first = nullptr, *count = nullptr;
    double* dbuf = nullptr;    // 8 x ninst
    int* ibuf = nullptr;       // 4 x ninst
    unsigned* tickets = nullptr;
    double* part = nullptr;    // 5 x nchunks
    double* norms = nullptr;   // 5 x ninst
    int* flag_a = nullptr;     // per-instance flag vectors (ninst each)
    int* flag_b = nullptr;
    std::vector<int> h_done, h_iters, h_status;
    std::vector<double> h_norms;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    float* dcomp = nullptr;    // FP32 K mode: the compensated diagonal's correction (n)

    Tables tables() const { return Tables{row0, row1, inst, first, count}; }
    Scalars scalars() const {
        Scalars S;
        const int n = ninst;
        S.rhs2 = dbuf;
        S.thr = dbuf + n;
        S.absnew = dbuf + 2 * n;
        S.pq = dbuf + 3 * n;
        S.alpha = dbuf + 4 * n;
        S.rr = dbuf + 5 * n;
        S.beta = dbuf + 6 * n;
        S.rrcap = dbuf + 7 * n;
        S.iters = ibuf;
        S.done = ibuf + n;
        S.status = ibuf + 2 * n;
        S.maxit = ibuf + 3 * n;
        S.ticket = tickets;
        S.ninst = n;
        S.timing = 0;
        return S;
    }
};

void batch_release(BatchState* b) {
    if (!b) return;
    for (cudaGraphExec_t g : b->graph)
        if (g) cudaGraphExecDestroy(g);
    void* ptrs[] = {b->row0, b->row1,    b->inst, b->first, b->count,  b->dbuf,
                    b->ibuf, b->tickets, b->part, b->norms, b->flag_a, b->flag_b, b->dcomp};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete b;
}

// Cut the block rows of every instance into chunks of at most R rows.
int batch_setup(nb2_ctx* c, const int* node_offsets, int ninst, int R, int lanes,
                BatchState** out) {
    *out = nullptr;
    if (ninst <= 0 || R <= 0 || node_offsets[0] != 0 || node_offsets[ninst] != c->N) {
        c->error = "instance node offsets must start at 0, increase, and end at the node count";
        return NB2_E_INPUT;
    }
    for (int i = 0; i < ninst; ++i)
        if (node_offsets[i + 1] <= node_offsets[i]) {
            c->error = "instance node offsets must increase";
            return NB2_E_INPUT;
        }
    auto* b = new BatchState();
    b->ninst = ninst;
    b->rows = R;
    b->lanes = lanes;
    b->h_node_off.assign(node_offsets, node_offsets + ninst + 1);
    std::vector<int> r0, r1, in;
    for (int i = 0; i < ninst; ++i) {
        b->h_first.push_back((int)r0.size());
        for (int a = node_offsets[i]; a < node_offsets[i + 1]; a += R) {
            r0.push_back(a);
            r1.push_back(std::min(a + R, node_offsets[i + 1]));
            in.push_back(i);
        }
        b->h_count.push_back((int)r0.size() - b->h_first.back());
    }
    b->nchunks = (int)r0.size();
    auto upload = [&](int** d, const std::vector<int>& h) -> cudaError_t {
        cudaError_t e = cudaMalloc(d, sizeof(int) * h.size());
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(*d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice,
                                c->stream);
        return e;
    };
    cudaError_t e = upload(&b->row0, r0);
    if (e == cudaSuccess) e = upload(&b->row1, r1);
    if (e == cudaSuccess) e = upload(&b->inst, in);
    if (e == cudaSuccess) e = upload(&b->first, b->h_first);
    if (e == cudaSuccess) e = upload(&b->count, b->h_count);
    if (e == cudaSuccess) e = cudaMalloc(&b->dbuf, sizeof(double) * 8 * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->ibuf, sizeof(int) * 4 * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->tickets, sizeof(unsigned) * 4 * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->part, sizeof(double) * 5 * b->nchunks);
    if (e == cudaSuccess) e = cudaMalloc(&b->norms, sizeof(double) * 5 * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->flag_a, sizeof(int) * ninst);
    if (e == cudaSuccess) e = cudaMalloc(&b->flag_b, sizeof(int) * ninst);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->dbuf, 0, sizeof(double) * 7 * ninst, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->ibuf, 0, sizeof(int) * 4 * ninst, c->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(b->tickets, 0, sizeof(unsigned) * 4 * ninst, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        batch_release(b);
        return cuda_fail(c, e, "batch_setup");
    }
    b->h_done.resize(ninst);
    b->h_iters.resize(ninst);
    b->h_status.resize(ninst);
    b->h_norms.resize(5 * ninst);
    *out = b;
    return NB2_OK;
}

int upload_flags(nb2_ctx* c, int* d, const std::vector<int>& h) {
    NB2_CUDA(c, cudaMemcpyAsync(d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice,
                                c->stream));
    return NB2_OK;
}

// per-instance norms of up to five vectors into b->h_norms[k * ninst + i] (synchronises)
int batch_norms(nb2_ctx* c, BatchState* b, const double* v0, const double* v1, const double* v2,
                const double* v3, const double* v4) {
    k_b_norms<<<b->nchunks, kThreads, 0, c->stream>>>(b->tables(), v0, v1, v2, v3, v4,
                                                      b->scalars(), b->part, b->norms);
    c->launches++;
    NB2_CUDA(c, cudaMemcpyAsync(b->h_norms.data(), b->norms, sizeof(double) * 5 * b->ninst,
                                cudaMemcpyDeviceToHost, c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

// Per-instance Jacobi-PCG on the resident K: kModeK64 (FP64 K) or kModeK32V64 (FP32 K); FP64
// vectors and dot products in both.  Instance i stops at its own tolerance or
// after maxit[i] iterations; an instance with b = 0 returns x = 0 at once.
//   batch_pcg_start    Jacobi inverse, x = 0, r = b, p = D^-1 r, per-instance thresholds
//   batch_pcg_iterate  captured blocks of iterations until every instance is done
int batch_pcg_start(nb2_ctx* c, BatchState* b, int mode, const double* rhs, double tol,
                    const std::vector<int>& maxit) {
    const Tables T = b->tables();
    const Scalars S = b->scalars();
    const unsigned g = (c->N + 255) / 256;
    if (mode == kModeK64)
        k_b_invdiag<double, double><<<g, 256, 0, c->stream>>>(c->brp, c->bcol, c->K64, c->N,
                                                              c->cg_inv);
    else {
        if (!b->dcomp) NB2_CUDA(c, cudaMalloc(&b->dcomp, sizeof(float) * c->n));
        k_b_compdiag<<<g, 256, 0, c->stream>>>(c->brp, c->bcol, c->K32, c->N, b->dcomp,
                                               c->cg_inv);
    }
    NB2_CUDA(c, cudaMemcpyAsync(S.maxit, maxit.data(), sizeof(int) * b->ninst,
                                cudaMemcpyHostToDevice, c->stream));
    k_b_init<double><<<b->nchunks, kThreads, 0, c->stream>>>(T, rhs, c->cg_x, c->cg_r, c->cg_p,
                                                              c->cg_inv, S, b->part, tol);
    c->launches += 2;
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));  // maxit's host vector is the caller's
    return NB2_OK;
}

int batch_pcg_iterate(nb2_ctx* c, BatchState* b, int mode, int most, bool graphs) {
    const Tables T = b->tables();
    const Scalars S = b->scalars();
    const int nb = b->nchunks;
    const auto spmv64 = spmv_variant<double, double>(b->lanes);
    const auto spmv3264 = spmv_variant<float, double>(b->lanes);
    auto enqueue = [&]() {
        for (int it = 0; it < kBatchChunk; ++it) {
            if (mode == kModeK64)
                spmv64<<<nb, kThreads, 0, c->stream>>>(T, c->brp, c->bcol, c->K64, c->cg_p,
                                                       c->cg_q, c->mask, S, b->part, nullptr);
            else
                spmv3264<<<nb, kThreads, 0, c->stream>>>(T, c->brp, c->bcol, c->K32, c->cg_p,
                                                         c->cg_q, c->mask, S, b->part, b->dcomp);
            k_b_xr<double><<<nb, kThreads, 0, c->stream>>>(T, c->cg_x, c->cg_r, c->cg_p, c->cg_q,
                                                           c->cg_inv, S, b->part);
            k_b_p<double><<<nb, kThreads, 0, c->stream>>>(T, c->cg_p, c->cg_r, c->cg_inv, S);
        }
    };
    cudaGraphExec_t& g = b->graph[mode];
    if (graphs && g == nullptr) {
        cudaGraph_t gr = nullptr;
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            enqueue();
            if (cudaStreamEndCapture(c->stream, &gr) == cudaSuccess && gr) {
                if (cudaGraphInstantiate(&g, gr, 0) != cudaSuccess) g = nullptr;
                cudaGraphDestroy(gr);
            }
        }
        cudaGetLastError();
    }
    const bool use_graph = graphs && g != nullptr;
    int guard = 0;
    for (;;) {
        NB2_CUDA(c, cudaMemcpyAsync(b->h_done.data(), S.done, sizeof(int) * b->ninst,
                                    cudaMemcpyDeviceToHost, c->stream));
        NB2_CUDA(c, cudaStreamSynchronize(c->stream));
        bool all = true;
        for (int v : b->h_done) all = all && v;
        if (all) break;
        if (++guard > most / kBatchChunk + 4) {
            c->error = "batched PCG did not stop within its iteration limit";
            return NB2_E_TIMEOUT;
        }
        if (use_graph)
            NB2_CUDA(c, cudaGraphLaunch(g, c->stream));
        else
            enqueue();
        c->launches += 3 * kBatchChunk;
    }
    NB2_CUDA(c, cudaMemcpyAsync(b->h_iters.data(), S.iters, sizeof(int) * b->ninst,
                                cudaMemcpyDeviceToHost, c->stream));
    NB2_CUDA(c, cudaMemcpyAsync(b->h_status.data(), S.status, sizeof(int) * b->ninst,
                                cudaMemcpyDeviceToHost, c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

// the whole FP64 solve: start, iterate, x out
int batch_pcg(nb2_ctx* c, BatchState* b, int mode, const double* rhs, double* xout,
              double tol, const std::vector<int>& maxit, bool graphs) {
    NB2_TRY(batch_pcg_start(c, b, mode, rhs, tol, maxit));
    NB2_TRY(batch_pcg_iterate(c, b, mode, *std::max_element(maxit.begin(), maxit.end()),
                              graphs));
    k_b_out<double><<<vgrid(c->n), 256, 0, c->stream>>>(c->n, c->cg_x, xout);
    c->launches++;
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

// ---------------------------------------------------------------------------------------
// Batched Newton: every instance runs static_matrix::solve / perform_equilibrium_iterations
// (static_matrix.hpp:145-187, 402-467) as a state machine; one round = one element pass and at
// most one linear solve for every instance that is still loading.
//   FRESH   start of a load increment at the last converged displacement (k = 0: f_ext, mask,
//           prescribed increment, lifting)
//   ITER    Newton iteration k >= 1
//   VERIFY  converged; the next element pass updates at the new displacement (neon's
//           update_internal_variables after convergence) and, if that succeeds, commits
// A failure (element status, CG, iteration limit) cuts the instance's increment back
// (adaptive_time_step.cpp:130-165) and restarts it from the last converged displacement.
// ---------------------------------------------------------------------------------------
enum Phase : int { P_FRESH = 0, P_ITER = 1, P_VERIFY = 2, P_DONE = 3, P_FAILED = 4 };

struct Inst {
    AdaptiveTimeStep load;
    int phase = P_FRESH;
    int k = 0;
    double norm_initial_residual = 1.0;
    long long newton = 0, cg = 0;
    int status = NB2_OK;
    std::string message;
    std::vector<nb2_newton_log> log;
};

struct Table {
    TimeTable table;
    int inst = 0;
};

int flags_to_status(unsigned f) {
    if (f & (1u << (NB2_E_NEG_DETJ - 1))) return NB2_E_NEG_DETJ;
    if (f & (1u << (NB2_E_RETURN_MAP - 1))) return NB2_E_RETURN_MAP;
    return NB2_E_NAN;
}

const char* status_message(int st) {
    switch (st) {
        case NB2_E_NEG_DETJ: return "Positive Jacobian assumption violated";
        case NB2_E_RETURN_MAP: return "Non-convergence in radial return method.";
        case NB2_E_NAN: return "Floating point error reported";
        case NB2_E_CG_MAXIT: return "Conjugate gradient solver maximum iterations reached";
        case NB2_E_NEWTON_MAXIT: return "Reached Newton-Raphson iteration limit";
        default: return "";
    }
}

bool any(const std::vector<int>& v) {
    return std::any_of(v.begin(), v.end(), [](int x) { return x != 0; });
}

struct DeviceBuffers {
    std::vector<void*> owned;
    template <typename T>
    int alloc(nb2_ctx* c, T** p, long long count) {
        NB2_CUDA(c, cudaMalloc((void**)p, sizeof(T) * std::max<long long>(count, 1)));
        owned.push_back(*p);
        return NB2_OK;
    }
    template <typename T>
    int upload(nb2_ctx* c, T** p, const std::vector<T>& h) {
        NB2_TRY(alloc(c, p, (long long)h.size()));
        if (!h.empty())
            NB2_CUDA(c, cudaMemcpyAsync(*p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice,
                                        c->stream));
        return NB2_OK;
    }
    ~DeviceBuffers() {
        for (void* p : owned) cudaFree(p);
    }
};

struct BatchNewton {
    nb2_ctx* c = nullptr;
    BatchState* b = nullptr;
    nb2_solver_options o{};
    int ninst = 0;
    std::vector<Inst> in;
    std::vector<Table> dir, frc;
    DeviceBuffers mem;
    int *d_dofs = nullptr, *d_dtab = nullptr, *d_don = nullptr;
    double* d_ddelta = nullptr;
    int *f_dofs = nullptr, *f_tab = nullptr, *f_on = nullptr;
    double *f_w = nullptr, *f_val = nullptr;
    int m_dir = 0, m_frc = 0;
    int *e_inst = nullptr, *on = nullptr;
    unsigned* iflags = nullptr;
    double* yvec = nullptr;  // FP64 product of the residual replacements (mixed)
    std::vector<unsigned> h_iflags;
    double t_elem = 0, t_solve = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    ~BatchNewton() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        batch_release(b);
    }

    bool mixed() const { return o.precision == NB2_MIXED; }

    void time_begin() { cudaEventRecord(ev0, c->stream); }
    double time_end() {
        cudaEventRecord(ev1, c->stream);
        cudaEventSynchronize(ev1);
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        return ms * 1e-3;
    }

    int upload_tables(const nb2_dof_table* t, const int32_t* offsets, std::vector<Table>& out,
                      bool weighted) {
        std::vector<int> dofs, tab;
        std::vector<double> w;
        bool any_w = false;
        for (int i = 0; i < ninst; ++i) {
            for (int j = offsets[i]; j < offsets[i + 1]; ++j) {
                const nb2_dof_table& d = t[j];
                if (d.num_points < 1 || d.num_dofs < 0 || (d.num_dofs > 0 && !d.dofs) ||
                    !d.times || !d.values) {
                    c->error = "invalid dof table";
                    return NB2_E_INPUT;
                }
                const int lo = 3 * b->h_node_off[i], hi = 3 * b->h_node_off[i + 1];
                for (int k = 0; k < d.num_dofs; ++k) {
                    if (d.dofs[k] < lo || d.dofs[k] >= hi) {
                        c->error = "a dof table refers to a dof outside its instance";
                        return NB2_E_INPUT;
                    }
                    dofs.push_back(d.dofs[k]);
                    tab.push_back((int)out.size());
                    w.push_back(weighted && d.weights ? d.weights[k] : 1.0);
                    any_w = any_w || (weighted && d.weights);
                }
                Table tb;
                tb.table.t.assign(d.times, d.times + d.num_points);
                tb.table.v.assign(d.values, d.values + d.num_points);
                tb.inst = i;
                out.push_back(std::move(tb));
            }
        }
        if (weighted) {
            m_frc = (int)dofs.size();
            NB2_TRY(mem.upload(c, &f_dofs, dofs));
            NB2_TRY(mem.upload(c, &f_tab, tab));
            if (any_w) NB2_TRY(mem.upload(c, &f_w, w));
            NB2_TRY(mem.alloc(c, &f_on, (long long)out.size()));
            NB2_TRY(mem.alloc(c, &f_val, (long long)out.size()));
        } else {
            m_dir = (int)dofs.size();
            NB2_TRY(mem.upload(c, &d_dofs, dofs));
            NB2_TRY(mem.upload(c, &d_dtab, tab));
            NB2_TRY(mem.alloc(c, &d_don, (long long)out.size()));
            NB2_TRY(mem.alloc(c, &d_ddelta, (long long)out.size()));
        }
        return NB2_OK;
    }

    void fail(int i, int st, std::vector<int>& reset) {
        Inst& s = in[i];
        s.status = st;
        s.message = status_message(st);
        if (!s.load.update(false)) {
            s.phase = P_FAILED;
            s.status = NB2_E_CUTBACK_LIMIT;
            s.message = "Too many reductions.  Convergence not judged likely";
            return;
        }
        s.phase = P_FRESH;
        s.k = 0;
        reset[i] = 1;  // displacement <- last converged displacement
    }

    // Per-instance mixed precision with reliable updates (the batched counterpart of
    // pcg_reliable_mixed): iterations on the FP32 K32 (its diagonal compensated, k_b_compdiag)
    // with FP64 vectors -- K32 carries most of the bytes, and FP32 vector recurrences cost more
    // iterations than they save on these nearly incompressible tet4 systems -- and when every
    // instance has paused (its recursive residual fell by delta) or finished, the paused ones get the true residual b - K x with the FP64
    // tangent (matrix-free, stored coefficients, only their elements) and continue with it,
    // keeping their search directions.
    int solve_mixed(const std::vector<int>& solving, std::vector<int>& its, std::vector<int>& st) {
        const Tables T = b->tables();
        const Scalars S = b->scalars();
        const double tol = o.cg_tolerance, delta = o.mixed_inner_tolerance;
        const int maxit = o.cg_maximum_iterations;
        NB2_CUDA(c, cudaMemsetAsync(b->norms, 0, sizeof(double) * ninst, c->stream));
        std::vector<int> mx(ninst, maxit);
        NB2_TRY(batch_pcg_start(c, b, kModeK32V64, c->rhs, std::max(tol, delta), mx));
        std::vector<double> b2(ninst), thr(ninst), thr_final(ninst), rr(ninst);
        NB2_CUDA(c, cudaMemcpyAsync(b2.data(), S.rhs2, sizeof(double) * ninst,
                                    cudaMemcpyDeviceToHost, c->stream));
        NB2_CUDA(c, cudaMemcpyAsync(thr.data(), S.thr, sizeof(double) * ninst,
                                    cudaMemcpyDeviceToHost, c->stream));
        NB2_CUDA(c, cudaStreamSynchronize(c->stream));
        std::vector<int> finished(ninst), paused(ninst), done(ninst), fresh_p(ninst), resets(ninst);
        for (int i = 0; i < ninst; ++i) {
            thr_final[i] = std::max(tol * tol * b2[i], DBL_MIN);
            finished[i] = !solving[i] || b2[i] == 0.0;
            its[i] = 0;
            st[i] = NB2_OK;
        }
        for (int update = 0; update < 1000; ++update) {
            NB2_TRY(batch_pcg_iterate(c, b, kModeK32V64, maxit, o.use_graphs != 0));
            for (int i = 0; i < ninst; ++i) {
                paused[i] = 0;
                fresh_p[i] = 0;
                if (finished[i]) continue;
                its[i] = b->h_iters[i];
                const int s = b->h_status[i];
                if (s == NB2_E_CG_BREAKDOWN && resets[i] < 3) {
                    // the cycle diverged (its retained search direction no longer fits the
                    // replaced residual): replace the residual again and restart the cycle
                    // with p = M^-1 r
                    ++resets[i];
                    fresh_p[i] = 1;
                    paused[i] = 1;
                } else if (s != NB2_OK && s != NB2_E_CG_MAXIT) {
                    st[i] = s;
                    finished[i] = 1;
                    if (std::getenv("NB2_DEBUG"))
                        std::fprintf(stderr, "[nb2] batch mixed CG: instance %d status %d after %d "
                                     "iterations (reliable update %d)\n", i, s, its[i], update);
                } else {
                    paused[i] = 1;
                }
            }
            if (!any(paused)) break;
            NB2_TRY(upload_flags(c, b->flag_a, paused));
            const int* on_before = c->inst_on;
            c->inst_on = b->flag_a;  // the FP64 product over the paused instances' elements only
            const int ap = launch_apply(c, c->cg_x, yvec);
            c->inst_on = on_before;
            NB2_TRY(ap);
            k_b_true_residual<double><<<b->nchunks, kThreads, 0, c->stream>>>(
                T, b->flag_a, c->rhs, yvec, c->mask, c->cg_inv, c->cg_r, S, b->part, b->norms);
            c->launches++;
            NB2_CUDA(c, cudaMemcpyAsync(rr.data(), b->norms, sizeof(double) * ninst,
                                        cudaMemcpyDeviceToHost, c->stream));
            NB2_CUDA(c, cudaStreamSynchronize(c->stream));
            bool restart = false;
            for (int i = 0; i < ninst; ++i) {
                done[i] = 1;
                if (!paused[i]) continue;
                if (!std::isfinite(rr[i])) {
                    st[i] = NB2_E_NAN;
                    finished[i] = 1;
                } else if (rr[i] < thr_final[i]) {
                    finished[i] = 1;
                } else if (its[i] >= maxit) {
                    st[i] = NB2_E_CG_MAXIT;
                    finished[i] = 1;
                } else {
                    thr[i] = std::max(thr_final[i], delta * delta * rr[i]);
                    done[i] = 0;
                    restart = true;
                }
            }
            if (std::getenv("NB2_DEBUG")) {
                int np = 0, nr = 0, mi = 0;
                double worst = 0.0;
                for (int i = 0; i < ninst; ++i) {
                    np += paused[i];
                    nr += !done[i];
                    mi = std::max(mi, its[i]);
                    if (paused[i] && thr_final[i] > 0) worst = std::max(worst, rr[i] / thr_final[i]);
                }
                std::fprintf(stderr, "[nb2] batch reliable update %d: paused %d restarted %d max its %d "
                             "worst rr/thr %.3e\n", update, np, nr, mi, worst);
            }
            if (!restart) break;
            NB2_CUDA(c, cudaMemcpyAsync(S.thr, thr.data(), sizeof(double) * ninst,
                                        cudaMemcpyHostToDevice, c->stream));
            NB2_CUDA(c, cudaMemcpyAsync(S.done, done.data(), sizeof(int) * ninst,
                                        cudaMemcpyHostToDevice, c->stream));
            if (any(fresh_p)) {
                NB2_TRY(upload_flags(c, b->flag_b, fresh_p));
                k_b_restart_cycle<<<(ninst + 255) / 256, 256, 0, c->stream>>>(ninst, b->flag_b, S);
                c->launches++;
            }
            k_b_p<double><<<b->nchunks, kThreads, 0, c->stream>>>(T, c->cg_p, c->cg_r, c->cg_inv,
                                                                  S);
            c->launches++;
            NB2_CUDA(c, cudaStreamSynchronize(c->stream));  // host vectors above
        }
        for (int i = 0; i < ninst; ++i)
            if (!finished[i]) st[i] = NB2_E_CG_MAXIT;
        k_b_out<double><<<vgrid(c->n), 256, 0, c->stream>>>(c->n, c->cg_x, c->du);
        c->launches++;
        return NB2_OK;
    }

    int solve_fp64(const std::vector<int>& solving, std::vector<int>& its, std::vector<int>& st) {
        std::vector<int> mx(ninst, o.cg_maximum_iterations);
        NB2_TRY(batch_pcg(c, b, kModeK64, c->rhs, c->du, o.cg_tolerance, mx, o.use_graphs != 0));
        for (int i = 0; i < ninst; ++i) {
            its[i] = solving[i] ? b->h_iters[i] : 0;
            st[i] = solving[i] ? b->h_status[i] : NB2_OK;
        }
        return NB2_OK;
    }

    // f_ext, the Dirichlet mask and the prescribed increment of the instances starting a load
    // increment (static_matrix.hpp:205-241, 322-351)
    int start_increments(const std::vector<int>& fresh) {
        const Tables T = b->tables();
        std::vector<int> dir_on(dir.size()), frc_on(frc.size());
        std::vector<double> dir_delta(dir.size()), frc_val(frc.size());
        for (size_t t = 0; t < dir.size(); ++t) {
            const Inst& s = in[dir[t].inst];
            const double time = s.load.step_time();
            dir_on[t] = fresh[dir[t].inst] && dir[t].table.active(time);
            dir_delta[t] = dir_on[t] ? dir[t].table.value(time) -
                                           dir[t].table.value(s.load.last_converged_time)
                                     : 0.0;
        }
        for (size_t t = 0; t < frc.size(); ++t) {
            const Inst& s = in[frc[t].inst];
            frc_on[t] = fresh[frc[t].inst];
            frc_val[t] = frc_on[t] ? frc[t].table.value(s.load.step_time()) : 0.0;
        }
        NB2_TRY(upload_flags(c, b->flag_a, fresh));
        k_b_fill<unsigned char><<<b->nchunks, kThreads, 0, c->stream>>>(T, b->flag_a, 1, c->mask,
                                                                         (unsigned char)0);
        k_b_fill<double><<<b->nchunks, kThreads, 0, c->stream>>>(T, b->flag_a, 1, c->fext, 0.0);
        NB2_CUDA(c, cudaMemsetAsync(c->inc, 0, sizeof(double) * c->n, c->stream));
        c->launches += 2;
        if (m_dir > 0) {
            NB2_TRY(upload_flags(c, d_don, dir_on));
            NB2_CUDA(c, cudaMemcpyAsync(d_ddelta, dir_delta.data(), sizeof(double) * dir.size(),
                                        cudaMemcpyHostToDevice, c->stream));
            k_b_dirichlet<<<(m_dir + 255) / 256, 256, 0, c->stream>>>(m_dir, d_dofs, d_dtab, d_don,
                                                                      d_ddelta, c->mask, c->inc);
            c->launches++;
        }
        if (m_frc > 0) {
            NB2_TRY(upload_flags(c, f_on, frc_on));
            NB2_CUDA(c, cudaMemcpyAsync(f_val, frc_val.data(), sizeof(double) * frc.size(),
                                        cudaMemcpyHostToDevice, c->stream));
            k_b_forces<<<(m_frc + 255) / 256, 256, 0, c->stream>>>(m_frc, f_dofs, f_tab, f_w, f_on,
                                                                   f_val, c->fext);
            c->launches++;
        }
        // the host vectors above must outlive the asynchronous copies
        NB2_CUDA(c, cudaStreamSynchronize(c->stream));
        return NB2_OK;
    }

    int run() {
        const Tables T = b->tables();
        const int prec = mixed() ? NB2_MIXED : NB2_FP64;
        const int mode =
            MODE_CONSTITUTIVE | MODE_STIFFNESS | MODE_FORCE | (mixed() ? MODE_STORE : 0);
        NB2_CUDA(c, cudaMemsetAsync(c->u, 0, sizeof(double) * c->n, c->stream));
        NB2_CUDA(c, cudaMemsetAsync(c->u_old, 0, sizeof(double) * c->n, c->stream));
        NB2_CUDA(c, cudaMemsetAsync(c->mask, 0, c->n, c->stream));
        std::vector<int> onv(ninst), solving(ninst), fresh(ninst), commit(ninst), reset(ninst);
        std::vector<int> its(ninst), cgst(ninst);
        long long rounds = 0;
        const long long round_limit = 1000000;
        for (;;) {
            for (int i = 0; i < ninst; ++i) onv[i] = in[i].phase <= P_VERIFY;
            if (!any(onv)) break;
            if (++rounds > round_limit) {
                c->error = "batched Newton did not finish";
                return NB2_E_TIMEOUT;
            }
            // element pass (update + tangent + f_int) for the instances still loading
            NB2_TRY(upload_flags(c, on, onv));
            NB2_CUDA(c, cudaMemsetAsync(iflags, 0, sizeof(unsigned) * ninst, c->stream));
            NB2_TRY(reset_status(c));
            time_begin();
            NB2_TRY(launch_element_kernel(c, mode, prec));
            t_elem += time_end();
            NB2_CUDA(c, cudaMemcpyAsync(h_iflags.data(), iflags, sizeof(unsigned) * ninst,
                                        cudaMemcpyDeviceToHost, c->stream));
            NB2_CUDA(c, cudaStreamSynchronize(c->stream));
            // decisions that need only the element pass
            std::fill(solving.begin(), solving.end(), 0);
            std::fill(fresh.begin(), fresh.end(), 0);
            std::fill(commit.begin(), commit.end(), 0);
            std::fill(reset.begin(), reset.end(), 0);
            for (int i = 0; i < ninst; ++i) {
                Inst& s = in[i];
                if (!onv[i]) continue;
                if (h_iflags[i]) {
                    fail(i, flags_to_status(h_iflags[i]), reset);
                    continue;
                }
                if (s.phase == P_VERIFY) {
                    commit[i] = 1;
                    s.load.update(true);
                    s.status = NB2_OK;
                    s.message.clear();
                    if (s.load.is_applied) {
                        s.phase = P_DONE;
                        continue;
                    }
                    s.phase = P_FRESH;
                    s.k = 0;
                }
                solving[i] = 1;
                fresh[i] = s.phase == P_FRESH;
            }
            if (any(commit)) {
                NB2_TRY(upload_flags(c, b->flag_a, commit));
                k_b_copy<<<b->nchunks, kThreads, 0, c->stream>>>(T, b->flag_a, c->u, c->u_old);
                c->launches++;
            }
            if (any(solving)) {
                const bool any_fresh = any(fresh);
                if (any_fresh) NB2_TRY(start_increments(fresh));
                // minus_residual = f_ext - f_int; lifting and the prescribed increment at k = 0
                k_b_sub<<<vgrid(c->n), 256, 0, c->stream>>>(c->n, c->fext, c->fint, c->rhs);
                c->launches++;
                if (any_fresh) {
                    double* tmp = c->cg_q;
                    if (mixed())
                        NB2_TRY(launch_apply(c, c->inc, tmp));
                    else
                        bsr_spmv_fp64(c, c->inc, tmp, false);
                    k_b_axpy<<<vgrid(c->n), 256, 0, c->stream>>>(c->n, -1.0, tmp, c->rhs);
                    k_b_axpy<<<vgrid(c->n), 256, 0, c->stream>>>(c->n, 1.0, c->inc, c->u);
                    c->launches += 2;
                    NB2_TRY(batch_norms(c, b, c->rhs, nullptr, nullptr, nullptr, nullptr));
                    for (int i = 0; i < ninst; ++i)
                        if (fresh[i]) in[i].norm_initial_residual = b->h_norms[i];
                }
                k_b_zero_masked<<<vgrid(c->n), 256, 0, c->stream>>>(c->n, c->mask, c->rhs);
                NB2_TRY(upload_flags(c, b->flag_b, solving));
                k_b_fill<double><<<b->nchunks, kThreads, 0, c->stream>>>(T, b->flag_b, 0, c->rhs,
                                                                          0.0);
                c->launches += 2;
                time_begin();
                NB2_TRY(mixed() ? solve_mixed(solving, its, cgst) : solve_fp64(solving, its, cgst));
                t_solve += time_end();
                k_b_axpy<<<vgrid(c->n), 256, 0, c->stream>>>(c->n, 1.0, c->du, c->u);
                c->launches++;
                NB2_TRY(batch_norms(c, b, c->du, c->u, c->rhs, c->fext, c->fint));
                const double* nv = b->h_norms.data();
                for (int i = 0; i < ninst; ++i) {
                    if (!solving[i]) continue;
                    Inst& s = in[i];
                    s.cg += its[i];
                    if (cgst[i] != NB2_OK) {
                        fail(i, cgst[i], reset);
                        continue;
                    }
                    // update_relative_norms (static_matrix.hpp:353-383)
                    const double du = nv[i], u = nv[ninst + i], r = nv[2 * ninst + i],
                                 fe = nv[3 * ninst + i], fi = nv[4 * ninst + i];
                    double dn = du, fn = r;
                    if (o.absolute_tolerance == 0 && !is_approx(u, 0.0, 1.0) &&
                        !is_approx(std::max(fe, fi), 0.0, 1.0)) {
                        dn = du / u;
                        fn = r / std::max(s.norm_initial_residual, std::max(fe, fi));
                    }
                    ++s.newton;
                    s.log.push_back({s.load.step_time(), s.k, its[i], dn, fn});
                    if (dn <= o.displacement_tolerance && fn <= o.residual_tolerance) {
                        s.phase = P_VERIFY;
                    } else if (++s.k == o.linear_iterations) {
                        fail(i, NB2_E_NEWTON_MAXIT, reset);
                    } else {
                        s.phase = P_ITER;
                    }
                }
            }
            if (any(reset)) {
                NB2_TRY(upload_flags(c, b->flag_a, reset));
                k_b_copy<<<b->nchunks, kThreads, 0, c->stream>>>(T, b->flag_a, c->u_old, c->u);
                c->launches++;
                NB2_CUDA(c, cudaStreamSynchronize(c->stream));
            }
        }
        NB2_CUDA(c, cudaStreamSynchronize(c->stream));
        NB2_CUDA(c, cudaGetLastError());
        return NB2_OK;
    }
};

}  // namespace

}  // namespace nb2

using namespace nb2;

extern "C" int nb2_batch_autotune(nb2_ctx* c, int32_t num_instances, const int32_t* node_offsets,
                                  int32_t precision, int32_t* rows_per_chunk,
                                  int32_t* lanes_per_row, double* ms_per_spmv) {
    if (!c || !node_offsets || num_instances <= 0) return NB2_E_INPUT;
    const bool f64 = precision == NB2_FP64;
    NB2_TRY(f64 ? ensure_k64(c) : ensure_k32(c));
    const int rows[] = {16, 32, 64, 128};
    const int lanes[] = {4, 8, 16, 32};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    NB2_CUDA(c, cudaEventCreate(&e0));
    NB2_CUDA(c, cudaEventCreate(&e1));
    double best = 1e30;
    int bestR = 32, bestL = 16;
    int st = NB2_OK;
    for (int R : rows) {
        BatchState* b = nullptr;
        st = batch_setup(c, node_offsets, num_instances, R, 16, &b);
        if (st) break;
        Scalars S = b->scalars();
        S.timing = 1;
        if (!f64 && cudaMalloc(&b->dcomp, sizeof(float) * c->n) == cudaSuccess)
            cudaMemsetAsync(b->dcomp, 0, sizeof(float) * c->n, c->stream);  // timed like the solve's
        for (int L : lanes) {
            auto sweep = [&]() {
                if (f64)
                    spmv_variant<double, double>(L)<<<b->nchunks, kThreads, 0, c->stream>>>(
                        b->tables(), c->brp, c->bcol, c->K64, c->cg_p, c->cg_q, c->mask, S,
                        b->part, nullptr);
                else  // the batched mixed mode: FP32 K, FP64 vectors
                    spmv_variant<float, double>(L)<<<b->nchunks, kThreads, 0, c->stream>>>(
                        b->tables(), c->brp, c->bcol, c->K32, c->cg_p, c->cg_q, c->mask, S,
                        b->part, b->dcomp);
            };
            sweep();
            cudaEventRecord(e0, c->stream);
            for (int k = 0; k < 5; ++k) sweep();
            cudaEventRecord(e1, c->stream);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            c->launches += 6;
            if (ms / 5 < best) {
                best = ms / 5;
                bestR = R;
                bestL = L;
            }
        }
        batch_release(b);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    NB2_CUDA(c, cudaGetLastError());
    c->batch_rows = bestR;
    c->batch_lanes = bestL;
    if (rows_per_chunk) *rows_per_chunk = bestR;
    if (lanes_per_row) *lanes_per_row = bestL;
    if (ms_per_spmv) *ms_per_spmv = best;
    return NB2_OK;
}

extern "C" int nb2_batch_static_solve(nb2_ctx* c, int32_t num_instances,
                                      const int32_t* node_offsets,
                                      const nb2_solver_options* options,
                                      const nb2_dof_table* dirichlet,
                                      const int32_t* dirichlet_offsets,
                                      const nb2_dof_table* nodal_forces,
                                      const int32_t* force_offsets, double* u_out,
                                      nb2_solve_report* reports, nb2_newton_log* log,
                                      int32_t max_log) {
    if (!c || !node_offsets || !options || num_instances <= 0 || !dirichlet_offsets ||
        !force_offsets || (dirichlet_offsets[num_instances] > 0 && !dirichlet) ||
        (force_offsets[num_instances] > 0 && !nodal_forces))
        return NB2_E_INPUT;
    if (c->mat.model == NB2_SMALL_STRAIN_J2_PLASTICITY) {
        c->error = "batched solves take models without history (no J2 plasticity)";
        return NB2_E_INPUT;
    }
    if (options->linear_iterations <= 0 || options->cg_maximum_iterations <= 0)
        return NB2_E_INPUT;
    for (int i = 0; i < num_instances; ++i)
        if (dirichlet_offsets[i + 1] < dirichlet_offsets[i] ||
            force_offsets[i + 1] < force_offsets[i])
            return NB2_E_INPUT;
    const auto t0 = std::chrono::steady_clock::now();
    c->error.clear();
    BatchNewton nw;
    nw.c = c;
    nw.o = *options;
    nw.ninst = num_instances;
    if (nw.mixed()) {
        NB2_TRY(ensure_k32(c));
        NB2_TRY(ensure_split_buffers(c));
        if (!(nw.o.mixed_inner_tolerance > 0)) nw.o.mixed_inner_tolerance = 1e-4;
    } else {
        NB2_TRY(ensure_k64(c));
    }
    const int R = c->batch_rows > 0 ? c->batch_rows : 32;
    const int L = c->batch_lanes > 0 ? c->batch_lanes : 16;
    NB2_TRY(batch_setup(c, node_offsets, num_instances, R, L, &nw.b));
    // element -> instance (and the check that no element couples two instances)
    int* d_off = nullptr;
    int* d_bad = nullptr;
    NB2_TRY(nw.mem.upload(c, &d_off,
                          std::vector<int>(node_offsets, node_offsets + num_instances + 1)));
    NB2_TRY(nw.mem.alloc(c, &d_bad, 1));
    NB2_TRY(nw.mem.alloc(c, &nw.e_inst, (long long)c->E));
    NB2_TRY(nw.mem.alloc(c, &nw.on, (long long)num_instances));
    NB2_TRY(nw.mem.alloc(c, &nw.iflags, (long long)num_instances));
    if (nw.mixed()) {
        NB2_TRY(nw.mem.alloc(c, &nw.yvec, (long long)c->n));
    }
    NB2_CUDA(c, cudaMemsetAsync(d_bad, 0, sizeof(int), c->stream));
    k_b_element_instance<<<(unsigned)((c->E + 255) / 256), 256, 0, c->stream>>>(
        c->E, c->npe, c->conn, d_off, num_instances, nw.e_inst, d_bad);
    c->launches++;
    int bad = 0;
    NB2_CUDA(c, cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    if (bad) {
        c->error = "an element couples nodes of two instances";
        return NB2_E_INPUT;
    }
    nw.h_iflags.resize(num_instances);
    NB2_TRY(nw.upload_tables(dirichlet, dirichlet_offsets, nw.dir, false));
    NB2_TRY(nw.upload_tables(nodal_forces, force_offsets, nw.frc, true));
    // per-instance load stepping over the union of its tables' times (static_matrix.hpp:109-143)
    nw.in.resize(num_instances);
    for (int i = 0; i < num_instances; ++i) {
        std::vector<double> history;
        for (auto* v : {&nw.dir, &nw.frc})
            for (auto& t : *v)
                if (t.inst == i) history.insert(history.end(), t.table.t.begin(), t.table.t.end());
        std::sort(history.begin(), history.end());
        history.erase(std::unique(history.begin(), history.end()), history.end());
        if (history.empty()) history = {0.0, options->period};
        nw.in[i].load.init(options->period, options->initial_increment, options->minimum_increment,
                           options->maximum_increment, options->adaptive != 0, history);
    }
    NB2_CUDA(c, cudaEventCreate(&nw.ev0));
    NB2_CUDA(c, cudaEventCreate(&nw.ev1));
    c->e_inst = nw.e_inst;
    c->inst_on = nw.on;
    c->inst_flags = nw.iflags;
    int st = nw.run();
    c->e_inst = nullptr;
    c->inst_on = nullptr;
    c->inst_flags = nullptr;
    if (u_out) {
        cudaMemcpyAsync(u_out, c->u, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess && st == NB2_OK) st = NB2_E_CUDA;
    }
    const double total =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    int first_failure = NB2_OK;
    for (int i = 0; i < num_instances; ++i) {
        const Inst& s = nw.in[i];
        const int status = st != NB2_OK ? st : (s.phase == P_DONE ? NB2_OK : s.status);
        if (status != NB2_OK && first_failure == NB2_OK) first_failure = status;
        if (reports) {
            nb2_solve_report& r = reports[i];
            r.status = status;
            r.load_steps = s.load.successful_increments;
            r.newton_iterations = s.newton;
            r.cg_iterations = s.cg;
            r.seconds_total = total;
            r.seconds_update_assembly = nw.t_elem;
            r.seconds_solve = nw.t_solve;
            std::snprintf(r.message, sizeof r.message, "%s",
                          st != NB2_OK ? c->error.c_str() : s.message.c_str());
        }
        if (log)
            for (int j = 0; j < (int)s.log.size() && j < max_log; ++j)
                log[(long long)i * max_log + j] = s.log[j];
    }
    if (st == NB2_OK && first_failure != NB2_OK && c->error.empty())
        c->error = "at least one instance failed (see its report)";
    return st != NB2_OK ? st : first_failure;
}
