// post.cu -- quadrature-point variables extrapolated and averaged to the nodes: the step after
// the solve that feeds neon's file output (mesh/mechanics/solid/mesh.cpp:174-214).
//
// neon (submesh::nodal_averaged_variable, submesh.cpp:271-344, and average_internal_variable,
// io/post/node_averaged_variables.hpp:18-41): element by element, each component's point values
// are extrapolated to the element's nodes with the shape function's extrapolation matrix E
// (shape_function.hpp:70-100) and added to the nodes, each addition counted; the nodal value is
// sum / count.  Here one thread per node walks the node's element slots (the node -> slot lists
// of the matrix-free operator, ascending element order -- the reference's summation order), so
// no atomics are needed and the result is deterministic.
//   hex8 (8 points): E = N^-1, N[l][a] = N_a(point l).  N is the Kronecker product of the 1-D
//   matrix M[p][n] = n_n(xi_p) (points -g, +g; nodes -1, +1), so E[a][l] = prod_d Minv[n_d(a)][p_d(l)]
//   with Minv = 1/g [[(1+g)/2, -(1-g)/2], [-(1-g)/2, (1+g)/2]], g = 1/sqrt(3).
//   tet4 (1 point): E = ones(4, 1) (tetrahedron.cpp:38-43).
#include <algorithm>
#include <cmath>

#include "nb2_internal.cuh"

namespace nb2 {

namespace {

struct Extrapolation {
    double E[8][8];  // [node][point]
};

Extrapolation hex8_extrapolation() {
    // corner a / point l signs in the reference order (hexahedron.cpp corners, Gauss points alike)
    const int s[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                         {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    const double g = 1.0 / std::sqrt(3.0);
    // Minv[n][p]: node n (0: -1, 1: +1), point p (0: -g, 1: +g)
    const double Minv[2][2] = {{(1.0 + g) / (2.0 * g), -(1.0 - g) / (2.0 * g)},
                               {-(1.0 - g) / (2.0 * g), (1.0 + g) / (2.0 * g)}};
    Extrapolation X;
    for (int a = 0; a < 8; ++a)
        for (int l = 0; l < 8; ++l) {
            double v = 1.0;
            for (int d = 0; d < 3; ++d) v *= Minv[s[a][d] > 0][s[l][d] > 0];
            X.E[a][l] = v;
        }
    return X;
}

// kind 0: symmetric tensor stored SoA [6][nqp] (11 22 33 23 13 12) -> 9 row-major components;
// kind 1: scalar [nqp]; kind 2: von Mises stress from the SoA Cauchy stress
__device__ __forceinline__ double point_value(const double* src, long long nqp, long long q,
                                              int kind, int c) {
    if (kind == 1) return src[q];
    if (kind == 2) {
        const double s0 = src[q], s1 = src[nqp + q], s2 = src[2 * nqp + q];
        const double s3 = src[3 * nqp + q], s4 = src[4 * nqp + q], s5 = src[5 * nqp + q];
        const double tr = (s0 + s1 + s2) / 3.0;
        const double d0 = s0 - tr, d1 = s1 - tr, d2 = s2 - tr;
        // stress_routines.hpp:19-36: sqrt(3/2) |dev sigma|
        return sqrt(1.5 * (d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * (s3 * s3 + s4 * s4 + s5 * s5)));
    }
    // row-major (i, j) -> Voigt slot: 00 0, 01 5, 02 4, 10 5, 11 1, 12 3, 20 4, 21 3, 22 2
    const int v = (c == 0) ? 0 : (c == 4) ? 1 : (c == 8) ? 2 : (c == 5 || c == 7) ? 3
                : (c == 2 || c == 6) ? 4 : 5;
    return src[v * nqp + q];
}

template <int NPE, int NQ>
__global__ void k_nodal_average(int N, const int* __restrict__ nptr, const int* __restrict__ nadj,
                                Extrapolation X, const double* __restrict__ src, long long nqp,
                                int kind, int nc, double* __restrict__ out) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= N) return;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int k0 = nptr[a], k1 = nptr[a + 1];
    for (int k = k0; k < k1; ++k) {
        const int slot = nadj[k];
        const long long e = slot / NPE;
        const int loc = slot - (int)e * NPE;
        for (int c = 0; c < nc; ++c) {
            double t = 0.0;
#pragma unroll
            for (int l = 0; l < NQ; ++l) t += X.E[loc][l] * point_value(src, nqp, e * NQ + l, kind, c);
            acc[c] += t;
        }
    }
    const double count = (double)(k1 - k0);
    for (int c = 0; c < nc; ++c) out[(long long)a * nc + c] = acc[c] / count;
}

}  // namespace

}  // namespace nb2

using namespace nb2;

extern "C" int nb2_nodal_averaged_variable(nb2_ctx* c, int32_t which, double* out) {
    if (!c || !out) return NB2_E_INPUT;
    const double* src = nullptr;
    int kind = 0, nc = 9;
    switch (which) {
        case 0: src = c->sig; kind = 0; nc = 9; break;
        case 1: src = c->detF; kind = 1; nc = 1; break;
        case 2: src = c->ep; kind = 0; nc = 9; break;
        case 3: src = c->epbar; kind = 1; nc = 1; break;
        case 4: src = c->sig; kind = 2; nc = 1; break;
        default: return NB2_E_INPUT;
    }
    if (!c->sig) {
        c->error = "nb2_nodal_averaged_variable needs a prior nb2_update_internal_variables";
        return NB2_E_INPUT;
    }
    if (!src) {  // plastic strains of a model without plasticity are zero
        std::fill(out, out + (size_t)c->N * nc, 0.0);
        return NB2_OK;
    }
    NB2_TRY(build_node_adjacency(c));
    Extrapolation X{};
    if (c->npe == 8) {
        X = hex8_extrapolation();
    } else {
        for (int a = 0; a < 4; ++a) X.E[a][0] = 1.0;
    }
    double* d_out = nullptr;
    NB2_CUDA(c, cudaMallocAsync(&d_out, sizeof(double) * (size_t)c->N * nc, c->stream));
    const unsigned grid = (unsigned)((c->N + 255) / 256);
    if (c->npe == 8)
        k_nodal_average<8, 8><<<grid, 256, 0, c->stream>>>(c->N, c->nadj_ptr, c->nadj, X, src,
                                                            c->nqp, kind, nc, d_out);
    else
        k_nodal_average<4, 1><<<grid, 256, 0, c->stream>>>(c->N, c->nadj_ptr, c->nadj, X, src,
                                                            c->nqp, kind, nc, d_out);
    c->launches++;
    NB2_CUDA(c, cudaGetLastError());
    NB2_CUDA(c, cudaMemcpyAsync(out, d_out, sizeof(double) * (size_t)c->N * nc,
                                cudaMemcpyDeviceToHost, c->stream));
    NB2_CUDA(c, cudaFreeAsync(d_out, c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}
