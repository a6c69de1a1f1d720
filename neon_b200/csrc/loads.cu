// loads.cu -- neon's non-follower loads (traction, pressure, body force) as nodal vectors per
// unit load value, computed on the device in the initial configuration.
//
// Reference path (dbeurle/neon):
//   nonfollower_load_boundary              src/mesh/mechanics/solid/boundary/nonfollower_load.cpp:12-121
//   surface_load::external_force (traction) src/mesh/boundary/neumann.hpp:69-133
//   pressure::external_force               src/mesh/mechanics/solid/boundary/pressure.cpp:9-37
//   volume_load::external_force (body force) src/mesh/boundary/neumann.hpp:135-192
//   quadrilateral4 / triangle3             src/interpolations/quadrilateral.cpp:17-45,
//                                          src/interpolations/triangle.cpp:16-40
//   surface rules                          src/quadrature/quadrilateral/quadrilateral_quadrature.cpp:5-24,
//                                          src/quadrature/triangle/triangle_quadrature.cpp:12-16 (x 0.5)
//   rule selection                         src/interpolations/interpolation_factory.cpp:99-117
//
// A load is linear in its time-table value and its geometry never moves, so each boundary is a
// fixed vector f times value(t); the Newton driver adds weights * value(t) into f_ext through
// its weighted DOF tables.  One thread per face (or element) writes the face's nodal
// contributions to its own slots; the node sums then run over the slots of each node in slot
// order, so the vector is the same on every run (no atomics).
#include <cmath>

#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/sort.h>

#include "nb2_internal.cuh"

namespace nb2 {

__constant__ double c_volume_dN[8 * 8 * 3];  // the context's element: dN at its points
__constant__ double c_volume_N[8 * 8];       // and N
__constant__ double c_volume_w[8];

// one thread per face: contributions [F][npf][3] of a traction (component comp) or a pressure
__global__ void k_surface_load(const double* __restrict__ X, const int* __restrict__ faces, int nf,
                               int npf, int kind, int comp, int reduced, double* __restrict__ out) {
    const int fc = blockIdx.x * blockDim.x + threadIdx.x;
    if (fc >= nf) return;
    const double g = 0.57735026918962576451;  // 1/sqrt(3)
    const double lq[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    int nq;
    double qx[4], qe[4], qw[4];
    if (npf == 4) {
        if (reduced) {
            nq = 1;
            qx[0] = 0.0, qe[0] = 0.0, qw[0] = 4.0;
        } else {
            nq = 4;
            for (int l = 0; l < 4; ++l) qx[l] = lq[l][0] * g, qe[l] = lq[l][1] * g, qw[l] = 1.0;
        }
    } else {
        nq = 1;
        qx[0] = 1.0 / 3.0, qe[0] = 1.0 / 3.0, qw[0] = 0.5;
    }
    double xa[4][3];
    for (int a = 0; a < npf; ++a)
        for (int i = 0; i < 3; ++i) xa[a][i] = X[3ll * faces[(size_t)fc * npf + a] + i];
    double fe[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int l = 0; l < nq; ++l) {
        double N[4], r[4][2];
        if (npf == 4) {
            for (int a = 0; a < 4; ++a) {
                N[a] = 0.25 * (1.0 + lq[a][0] * qx[l]) * (1.0 + lq[a][1] * qe[l]);
                r[a][0] = 0.25 * (1.0 + lq[a][1] * qe[l]) * lq[a][0];
                r[a][1] = 0.25 * (1.0 + lq[a][0] * qx[l]) * lq[a][1];
            }
        } else {
            N[0] = qx[l], N[1] = qe[l], N[2] = 1.0 - qx[l] - qe[l];
            r[0][0] = 1.0, r[0][1] = 0.0, r[1][0] = 0.0, r[1][1] = 1.0;
            r[2][0] = -1.0, r[2][1] = -1.0;
        }
        // the 3x2 surface Jacobian's columns, their cross product and its norm
        double t0[3] = {0, 0, 0}, t1[3] = {0, 0, 0};
        for (int a = 0; a < npf; ++a)
            for (int i = 0; i < 3; ++i) {
                t0[i] += xa[a][i] * r[a][0];
                t1[i] += xa[a][i] * r[a][1];
            }
        const double cr[3] = {t0[1] * t1[2] - t0[2] * t1[1], t0[2] * t1[0] - t0[0] * t1[2],
                              t0[0] * t1[1] - t0[1] * t1[0]};
        const double j = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        for (int a = 0; a < npf; ++a) {
            if (kind == NB2_LOAD_TRACTION)
                fe[a][comp] += N[a] * j * qw[l];
            else  // the unit normal times the surface measure, as neon forms it
                for (int i = 0; i < 3; ++i) fe[a][i] += N[a] * (cr[i] / j) * j * qw[l];
        }
    }
    const double sgn = kind == NB2_LOAD_PRESSURE ? -1.0 : 1.0;  // positive pressure compresses
    for (int a = 0; a < npf; ++a)
        for (int i = 0; i < 3; ++i) out[((size_t)fc * npf + a) * 3 + i] = sgn * fe[a][i];
}

// one thread per element: the body-force contribution sum_q w N_a det(X dN) of each node
template <int NPE>
__global__ void k_volume_load(const double* __restrict__ X, const int* __restrict__ conn, int E,
                              int nq, double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    double xa[NPE][3];
#pragma unroll
    for (int a = 0; a < NPE; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) xa[a][i] = X[3ll * conn[(size_t)e * NPE + a] + i];
    double fe[NPE];
#pragma unroll
    for (int a = 0; a < NPE; ++a) fe[a] = 0.0;
    for (int l = 0; l < nq; ++l) {
        double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) J[i * 3 + k] += xa[a][i] * c_volume_dN[(l * NPE + a) * 3 + k];
        const double j = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                         J[2] * (J[3] * J[7] - J[4] * J[6]);
#pragma unroll
        for (int a = 0; a < NPE; ++a) fe[a] += c_volume_N[l * NPE + a] * j * c_volume_w[l];
    }
#pragma unroll
    for (int a = 0; a < NPE; ++a) out[(size_t)e * NPE + a] = fe[a];
}

// node sums over slot lists sorted by node: the thread at the start of a node's run adds the
// run in slot order (per = values per slot: 3 for surfaces, 1 for volumes written to comp)
__global__ void k_gather_runs(long long m, const int* __restrict__ node_of, const int* __restrict__ slot,
                              const double* __restrict__ contrib, int per, int comp,
                              double* __restrict__ f) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m) return;
    const int nd = node_of[p];
    if (p > 0 && node_of[p - 1] == nd) return;
    double s[3] = {0.0, 0.0, 0.0};
    for (long long q = p; q < m && node_of[q] == nd; ++q)
        for (int i = 0; i < per; ++i) s[i] += contrib[(size_t)slot[q] * per + i];
    if (per == 3)
        for (int i = 0; i < 3; ++i) f[3ll * nd + i] = s[i];
    else
        f[3ll * nd + comp] = s[0];
}

__global__ void k_iota_slots(long long m, int* v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) v[i] = (int)i;
}

}  // namespace nb2

using namespace nb2;

extern "C" int nb2_nonfollower_load(nb2_ctx* c, int32_t kind, int32_t component,
                                    const int32_t* faces, int32_t num_faces,
                                    int32_t nodes_per_face, int32_t reduced_quadrature,
                                    double* f_out) {
    if (!c || !f_out) return NB2_E_INPUT;
    const bool surface = kind == NB2_LOAD_TRACTION || kind == NB2_LOAD_PRESSURE;
    if (!surface && kind != NB2_LOAD_BODY_FORCE) {
        c->error = "non-follower load: kind must be traction, pressure or body force";
        return NB2_E_INPUT;
    }
    if (kind != NB2_LOAD_PRESSURE && (component < 0 || component > 2)) {
        c->error = "non-follower load: component must be 0 (x), 1 (y) or 2 (z)";
        return NB2_E_INPUT;
    }
    long long m = 0;  // slots
    if (surface) {
        if (!faces || num_faces <= 0 || (nodes_per_face != 3 && nodes_per_face != 4)) {
            c->error = "non-follower load: surface loads need tri3 or quad4 faces";
            return NB2_E_INPUT;
        }
        m = (long long)num_faces * nodes_per_face;
        for (long long i = 0; i < m; ++i)
            if (faces[i] < 0 || faces[i] >= c->N) {
                c->error = "non-follower load: face node index out of range";
                return NB2_E_INPUT;
            }
    } else {
        m = (long long)c->E * c->npe;
        const double lc[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                 {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
        const double g = 1.0 / std::sqrt(3.0);
        double dN[8 * 8 * 3] = {0}, N[8 * 8] = {0}, w[8] = {0};
        if (c->npe == 8) {
            for (int l = 0; l < 8; ++l) {
                const double xi = lc[l][0] * g, eta = lc[l][1] * g, zeta = lc[l][2] * g;
                w[l] = 1.0;
                for (int a = 0; a < 8; ++a) {
                    const double xa = lc[a][0], ea = lc[a][1], za = lc[a][2];
                    N[l * 8 + a] = 0.125 * (1.0 + xa * xi) * (1.0 + ea * eta) * (1.0 + za * zeta);
                    dN[(l * 8 + a) * 3 + 0] = 0.125 * xa * (1.0 + ea * eta) * (1.0 + za * zeta);
                    dN[(l * 8 + a) * 3 + 1] = 0.125 * (1.0 + xa * xi) * ea * (1.0 + za * zeta);
                    dN[(l * 8 + a) * 3 + 2] = 0.125 * (1.0 + xa * xi) * (1.0 + ea * eta) * za;
                }
            }
        } else {
            const double dNt[12] = {1, 0, 0, 0, 1, 0, 0, 0, 1, -1, -1, -1};
            for (int i = 0; i < 12; ++i) dN[i] = dNt[i];
            for (int a = 0; a < 4; ++a) N[a] = 0.25;
            w[0] = 1.0 / 6.0;
        }
        NB2_CUDA(c, cudaMemcpyToSymbolAsync(c_volume_dN, dN, sizeof dN, 0, cudaMemcpyHostToDevice,
                                            c->stream));
        NB2_CUDA(c, cudaMemcpyToSymbolAsync(c_volume_N, N, sizeof N, 0, cudaMemcpyHostToDevice,
                                            c->stream));
        NB2_CUDA(c, cudaMemcpyToSymbolAsync(c_volume_w, w, sizeof w, 0, cudaMemcpyHostToDevice,
                                            c->stream));
    }
    const int per = surface ? 3 : 1;
    double* contrib = nullptr;
    double* f = nullptr;
    int *node_of = nullptr, *slot = nullptr, *dfaces = nullptr;
    int status = NB2_OK;
    auto fail = [&](cudaError_t e, const char* what) {
        status = cuda_fail(c, e, what);
        return status;
    };
#define LTRY(call)                                   \
    do {                                             \
        cudaError_t _e = (call);                     \
        if (_e != cudaSuccess) {                     \
            fail(_e, #call);                         \
            goto done;                               \
        }                                            \
    } while (0)
    {
        const int T = 256;
        const unsigned grid = (unsigned)((m + T - 1) / T);
        LTRY(cudaMallocAsync(&contrib, sizeof(double) * per * m, c->stream));
        LTRY(cudaMallocAsync(&f, sizeof(double) * c->n, c->stream));
        LTRY(cudaMallocAsync(&node_of, sizeof(int) * m, c->stream));
        LTRY(cudaMallocAsync(&slot, sizeof(int) * m, c->stream));
        LTRY(cudaMemsetAsync(f, 0, sizeof(double) * c->n, c->stream));
        if (surface) {
            LTRY(cudaMallocAsync(&dfaces, sizeof(int) * m, c->stream));
            LTRY(cudaMemcpyAsync(dfaces, faces, sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
            k_surface_load<<<(num_faces + T - 1) / T, T, 0, c->stream>>>(
                c->X, dfaces, num_faces, nodes_per_face, kind, component, reduced_quadrature,
                contrib);
            LTRY(cudaMemcpyAsync(node_of, dfaces, sizeof(int) * m, cudaMemcpyDeviceToDevice,
                                 c->stream));
        } else {
            const unsigned ge = (unsigned)((c->E + T - 1) / T);
            if (c->npe == 8)
                k_volume_load<8><<<ge, T, 0, c->stream>>>(c->X, c->conn, c->E, c->nq, contrib);
            else
                k_volume_load<4><<<ge, T, 0, c->stream>>>(c->X, c->conn, c->E, c->nq, contrib);
            LTRY(cudaMemcpyAsync(node_of, c->conn, sizeof(int) * m, cudaMemcpyDeviceToDevice,
                                 c->stream));
        }
        c->launches++;
        k_iota_slots<<<grid, T, 0, c->stream>>>(m, slot);
        // slots grouped by node, in slot order within a node (stable sort)
        thrust::stable_sort_by_key(thrust::cuda::par.on(c->stream),
                                   thrust::device_ptr<int>(node_of),
                                   thrust::device_ptr<int>(node_of) + m,
                                   thrust::device_ptr<int>(slot));
        k_gather_runs<<<grid, T, 0, c->stream>>>(m, node_of, slot, contrib, per, component, f);
        c->launches += 2;
        LTRY(cudaGetLastError());
        LTRY(cudaMemcpyAsync(f_out, f, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
        LTRY(cudaStreamSynchronize(c->stream));
    }
done:
#undef LTRY
    if (contrib) cudaFreeAsync(contrib, c->stream);
    if (f) cudaFreeAsync(f, c->stream);
    if (node_of) cudaFreeAsync(node_of, c->stream);
    if (slot) cudaFreeAsync(slot, c->stream);
    if (dfaces) cudaFreeAsync(dfaces, c->stream);
    cudaStreamSynchronize(c->stream);
    return status;
}
