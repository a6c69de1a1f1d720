// pattern.cu -- CSR sparsity pattern built once on the device, element->block slot map, and the
// block -> neon CSR value permutation used by the drop-in export.
//
// neon builds its pattern with Eigen setFromTriplets over every (dof_p, dof_q) pair of every
// element (src/assembler/sparsity_pattern.hpp:18-48), which gives per row the sorted unique set
// of coupled columns.  Every node pair sharing an element couples all 3x3 DOF pairs, so that
// pattern is exactly the node-block pattern expanded: here the node-pair keys are radix-sorted and
// de-duplicated on the device (brp/bcol), and CSR row 3*a+r lists, for each neighbour block b of
// node a in ascending order, the columns 3b, 3b+1, 3b+2.
#include <algorithm>
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/scan.h>
#include <thrust/sort.h>
#include <thrust/unique.h>

#include "nb2_internal.cuh"

namespace nb2 {

__global__ void k_emit_pairs(const int* __restrict__ conn, int E, int npe,
                             unsigned long long* __restrict__ keys) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)E * npe * npe;
    if (t >= total) return;
    int e = (int)(t / (npe * npe));
    int ab = (int)(t % (npe * npe));
    int a = ab / npe, b = ab % npe;
    unsigned long long na = (unsigned)conn[(long long)e * npe + a];
    unsigned long long nb = (unsigned)conn[(long long)e * npe + b];
    keys[t] = (na << 32) | nb;
}

__global__ void k_split_keys(const unsigned long long* __restrict__ keys, long long m,
                             int* __restrict__ row_count, int* __restrict__ bcol) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    unsigned long long k = keys[t];
    bcol[t] = (int)(k & 0xffffffffull);
    atomicAdd(&row_count[(int)(k >> 32)], 1);
}

// slot[e][a*npe+b] = index of block (conn[e][a], conn[e][b]) in bcol
__global__ void k_slot_map(const int* __restrict__ conn, int E, int npe, const int* __restrict__ brp,
                           const int* __restrict__ bcol, int* __restrict__ slot) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)E * npe * npe;
    if (t >= total) return;
    int e = (int)(t / (npe * npe));
    int ab = (int)(t % (npe * npe));
    int a = ab / npe, b = ab % npe;
    int na = conn[(long long)e * npe + a];
    int nb = conn[(long long)e * npe + b];
    int lo = brp[na], hi = brp[na + 1] - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (bcol[mid] < nb)
            lo = mid + 1;
        else
            hi = mid;
    }
    slot[t] = lo;
}

// CSR position of block s (row node a, k-th neighbour), entry (r, c):
//   9*brp[a] + r*3*deg(a) + 3k + c
__global__ void k_bsr_to_csr(const int* __restrict__ brp, int N, const double* __restrict__ Kb,
                             double* __restrict__ Kc) {
    int a = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    int lane = threadIdx.x & 31;
    if (a >= N) return;
    int b0 = brp[a], deg = brp[a + 1] - b0;
    long long base = 9ll * b0;
    for (int v = lane; v < 9 * deg; v += 32) {
        int k = v / 9, e = v - 9 * k, r = e / 3, cc = e - 3 * r;
        Kc[base + (long long)r * 3 * deg + 3 * k + cc] = Kb[base + v];
    }
}

int build_pattern(nb2_ctx* c) {
    const long long pairs = (long long)c->E * c->npe * c->npe;
    unsigned long long* keys = nullptr;
    NB2_CUDA(c, cudaMallocAsync(&keys, sizeof(unsigned long long) * pairs, c->stream));
    const int T = 256;
    k_emit_pairs<<<(unsigned)((pairs + T - 1) / T), T, 0, c->stream>>>(c->conn, c->E, c->npe, keys);
    c->launches++;
    auto pol = thrust::cuda::par.on(c->stream);
    thrust::device_ptr<unsigned long long> kp(keys);
    thrust::sort(pol, kp, kp + pairs);
    auto end = thrust::unique(pol, kp, kp + pairs);
    long long m = end - kp;
    if (9 * m > 2147483647ll) {
        // the CSR export (and neon's Eigen matrix) index entries with int32
        cudaFreeAsync(keys, c->stream);
        c->error = "the stiffness pattern has more than 2^31 - 1 entries: beyond the int32 row "
                   "pointers and column indices of the CSR matrix";
        return NB2_E_INPUT;
    }
    c->nnzb = m;
    c->nnz = 9 * m;
    int* count = nullptr;
    NB2_CUDA(c, cudaMallocAsync(&count, sizeof(int) * (c->N + 1), c->stream));
    NB2_CUDA(c, cudaMemsetAsync(count, 0, sizeof(int) * (c->N + 1), c->stream));
    NB2_CUDA(c, cudaMalloc(&c->bcol, sizeof(int) * m));
    NB2_CUDA(c, cudaMalloc(&c->brp, sizeof(int) * (c->N + 1)));
    k_split_keys<<<(unsigned)((m + T - 1) / T), T, 0, c->stream>>>(keys, m, count, c->bcol);
    c->launches++;
    thrust::device_ptr<int> cp(count), bp(c->brp);
    thrust::exclusive_scan(pol, cp, cp + c->N + 1, bp);
    NB2_CUDA(c, cudaMalloc(&c->slot, sizeof(int) * pairs));
    k_slot_map<<<(unsigned)((pairs + T - 1) / T), T, 0, c->stream>>>(c->conn, c->E, c->npe, c->brp,
                                                                       c->bcol, c->slot);
    c->launches++;
    NB2_CUDA(c, cudaFreeAsync(keys, c->stream));
    NB2_CUDA(c, cudaFreeAsync(count, c->stream));
    c->h_brp.resize(c->N + 1);
    c->h_bcol.resize(m);
    NB2_CUDA(c, cudaMemcpyAsync(c->h_brp.data(), c->brp, sizeof(int) * (c->N + 1),
                                cudaMemcpyDeviceToHost, c->stream));
    NB2_CUDA(c, cudaMemcpyAsync(c->h_bcol.data(), c->bcol, sizeof(int) * m, cudaMemcpyDeviceToHost,
                                c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

__global__ void k_iota(long long n, int* v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int)i;
}

// first position of each node in the node-sorted slot list (sorted keys: binary search)
__global__ void k_node_starts(const int* keys, long long m, int N, int* ptr) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a > N) return;
    long long lo = 0, hi = m;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (keys[mid] < a) lo = mid + 1; else hi = mid;
    }
    ptr[a] = (int)lo;
}

// For every node the element slots e*npe + a that reference it, in ascending slot order (a
// stable sort keeps it), so the matrix-free gather sums them in a fixed order.
int build_node_adjacency(nb2_ctx* c) {
    if (c->nadj) return NB2_OK;
    const long long m = (long long)c->E * c->npe;
    int* keys = nullptr;
    NB2_CUDA(c, cudaMallocAsync(&keys, sizeof(int) * m, c->stream));
    NB2_CUDA(c, cudaMalloc(&c->nadj, sizeof(int) * m));
    NB2_CUDA(c, cudaMalloc(&c->nadj_ptr, sizeof(int) * (c->N + 1)));
    NB2_CUDA(c, cudaMemcpyAsync(keys, c->conn, sizeof(int) * m, cudaMemcpyDeviceToDevice, c->stream));
    const int T = 256;
    k_iota<<<(unsigned)((m + T - 1) / T), T, 0, c->stream>>>(m, c->nadj);
    auto pol = thrust::cuda::par.on(c->stream);
    thrust::device_ptr<int> kp(keys), vp(c->nadj);
    thrust::stable_sort_by_key(pol, kp, kp + m, vp);
    k_node_starts<<<(c->N + 1 + T - 1) / T, T, 0, c->stream>>>(keys, m, c->N, c->nadj_ptr);
    c->launches += 2;
    NB2_CUDA(c, cudaFreeAsync(keys, c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

// Element colouring for the colour-partitioned launches (hex8, one problem).  Greedy first fit in
// element order over the node-sharing graph (a structured hex8 mesh gets the 8 parity colours);
// the elements are then listed colour by colour.  Not applicable (colour_state -1) to tet4 or
// when more than 64 colours would be needed.
int ensure_colouring(nb2_ctx* c) {
    if (c->colour_state != 0) return NB2_OK;
    if (c->npe != 8) {
        c->colour_state = -1;
        return NB2_OK;
    }
    NB2_TRY(build_node_adjacency(c));
    const int E = c->E, npe = c->npe, N = c->N;
    const long long m = (long long)E * npe;
    std::vector<int> conn(m), ptr(N + 1), adj(m);
    NB2_CUDA(c, cudaMemcpyAsync(conn.data(), c->conn, sizeof(int) * m, cudaMemcpyDeviceToHost,
                                c->stream));
    NB2_CUDA(c, cudaMemcpyAsync(ptr.data(), c->nadj_ptr, sizeof(int) * (N + 1),
                                cudaMemcpyDeviceToHost, c->stream));
    NB2_CUDA(c, cudaMemcpyAsync(adj.data(), c->nadj, sizeof(int) * m, cudaMemcpyDeviceToHost,
                                c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    std::vector<unsigned char> col(E);
    int ncol = 0;
    for (int e = 0; e < E; ++e) {
        unsigned long long used = 0ull;
        for (int a = 0; a < npe; ++a) {
            const int n = conn[(size_t)e * npe + a];
            for (int p = ptr[n]; p < ptr[n + 1]; ++p) {
                const int f = adj[p] / npe;
                if (f < e) used |= 1ull << col[f];
            }
        }
        if (used == ~0ull) {
            c->colour_state = -1;
            return NB2_OK;
        }
        const int k = __builtin_ctzll(~used);
        col[e] = (unsigned char)k;
        ncol = std::max(ncol, k + 1);
    }
    std::vector<int> coff(ncol + 1, 0), order(E);
    for (int e = 0; e < E; ++e) coff[col[e] + 1]++;
    for (int k = 0; k < ncol; ++k) coff[k + 1] += coff[k];
    std::vector<int> pos(coff.begin(), coff.end() - 1);
    for (int e = 0; e < E; ++e) order[pos[col[e]]++] = e;
    NB2_CUDA(c, cudaMalloc(&c->corder, sizeof(int) * E));
    NB2_CUDA(c, cudaMemcpyAsync(c->corder, order.data(), sizeof(int) * E, cudaMemcpyHostToDevice,
                                c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    c->h_coff = coff;
    c->colour_state = 1;
    return NB2_OK;
}

int export_csr_values(nb2_ctx* c, const double* Kbsr, double* Kcsr_dev) {
    const int T = 256;
    k_bsr_to_csr<<<(c->N + T / 32 - 1) / (T / 32), T, 0, c->stream>>>(c->brp, c->N, Kbsr, Kcsr_dev);
    c->launches++;
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

}  // namespace nb2
