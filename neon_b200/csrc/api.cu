// api.cu -- the C-ABI (include/neon_b200.h): context lifetime, element-level drop-ins, the
// linear-solver plugin and the static_matrix Newton driver over device-resident state.
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

int cuda_fail(nb2_ctx* c, cudaError_t e, const char* what) {
    if (c) c->error = std::string(what) + ": " + cudaGetErrorString(e);
    return NB2_E_CUDA;
}

static std::string g_create_error;

// ----- small vector kernels ---------------------------------------------------------------
__global__ void k_sub(long long n, const double* a, const double* b, double* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = a[i] - b[i];
}
__global__ void k_axpy(long long n, double alpha, const double* x, double* y) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] += alpha * x[i];
}
__global__ void k_zero_masked(long long n, const unsigned char* mask, double* v) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (mask[i]) v[i] = 0.0;
}
__global__ void k_scatter_set(int m, const int* dofs, double value, double* v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) v[dofs[i]] = value;
}
__global__ void k_scatter_mask(int m, const int* dofs, unsigned char* mask) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) mask[dofs[i]] = 1;
}
__global__ void k_scatter_add_weighted(int m, const int* dofs, const double* w, double value,
                                       double* v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) v[dofs[i]] += (w ? w[i] : 1.0) * value;
}
__global__ void k_sym6_to_9(long long nqp, const double* s6, double* out) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nqp) return;
    double a = s6[0 * nqp + q], b = s6[1 * nqp + q], c = s6[2 * nqp + q];
    double d = s6[3 * nqp + q], e = s6[4 * nqp + q], f = s6[5 * nqp + q];
    double* o = out + 9 * q;
    o[0] = a; o[1] = f; o[2] = e;
    o[3] = f; o[4] = b; o[5] = d;
    o[6] = e; o[7] = d; o[8] = c;
}

static unsigned grid_for(long long n) {
    long long g = (n + 255) / 256;
    return (unsigned)std::min<long long>(g, 148 * 8);
}

}  // namespace nb2

using namespace nb2;

// ---------------------------------------------------------------------------------------
// status word -> neon's computational_error messages
// ---------------------------------------------------------------------------------------
int nb2::reset_status(nb2_ctx* c) {
    DeviceStatus z{0u, 0u, ~0ull};
    NB2_CUDA(c, cudaMemcpyAsync(c->status, &z, sizeof z, cudaMemcpyHostToDevice, c->stream));
    return NB2_OK;
}

int nb2::read_status(nb2_ctx* c) {
    DeviceStatus h;
    NB2_CUDA(c, cudaMemcpyAsync(&h, c->status, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    if (h.flags == 0) return NB2_OK;
    if (h.flags & (1u << (NB2_E_NEG_DETJ - 1))) {
        unsigned long long q = h.negdet_first >> 32;
        unsigned bits = (unsigned)(h.negdet_first & 0xffffffffull);
        float v;
        std::memcpy(&v, &bits, sizeof v);
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "Positive Jacobian assumption violated at element %llu and local quadrature "
                      "point %llu (%g), another %u violations found",
                      q / c->nq, q % c->nq, (double)v, h.negdet_count - 1);
        c->error = buf;
        return NB2_E_NEG_DETJ;
    }
    if (h.flags & (1u << (NB2_E_RETURN_MAP - 1))) {
        c->error = "Non-convergence in radial return method.";
        return NB2_E_RETURN_MAP;
    }
    c->error = "Floating point error reported";
    return NB2_E_NAN;
}

template <typename T>
static int dev_alloc(nb2_ctx* c, T** p, long long count) {
    NB2_CUDA(c, cudaMalloc((void**)p, sizeof(T) * (count > 0 ? count : 1)));
    NB2_CUDA(c, cudaMemsetAsync(*p, 0, sizeof(T) * (count > 0 ? count : 1), c->stream));
    return NB2_OK;
}

int nb2::ensure_split_buffers(nb2_ctx* c) {
    if (c->sig) return NB2_OK;
    NB2_TRY(dev_alloc(c, &c->sig, 6ll * c->nqp));
    NB2_TRY(dev_alloc(c, &c->dpar, (long long)dpar_rows(c->mat.model) * c->nqp));
    NB2_TRY(dev_alloc(c, &c->detF, (long long)c->nqp));
    NB2_TRY(dev_alloc(c, &c->u_tan, (long long)c->n));
    return NB2_OK;
}

int nb2::ensure_k32(nb2_ctx* c) {
    NB2_TRY(ensure_cg32(c));
    if (c->K32) return NB2_OK;
    return dev_alloc(c, &c->K32, 9 * c->nnzb);
}

int nb2::ensure_cg32(nb2_ctx* c) {
    if (c->cg32_x) return NB2_OK;
    NB2_TRY(dev_alloc(c, &c->cg32_x, (long long)c->n));
    NB2_TRY(dev_alloc(c, &c->cg32_r, (long long)c->n));
    NB2_TRY(dev_alloc(c, &c->cg32_p, (long long)c->n));
    NB2_TRY(dev_alloc(c, &c->cg32_q, (long long)c->n));
    NB2_TRY(dev_alloc(c, &c->cg32_inv, (long long)c->n));
    return NB2_OK;
}

int nb2::ensure_k64(nb2_ctx* c) {
    if (c->K64) return NB2_OK;
    return dev_alloc(c, &c->K64, 9 * c->nnzb);
}

// The second FP64 K buffer for the double-buffered zeroing; when it does not fit, passes zero
// their K on the main stream instead (kalt_state -1)
int nb2::ensure_k64_alt(nb2_ctx* c) {
    if (c->kalt_state != 0) return NB2_OK;
    c->kalt_state = -1;
    if (cudaMalloc(&c->K64_alt, sizeof(double) * 9 * c->nnzb) != cudaSuccess) {
        cudaGetLastError();  // an allocation failure is not sticky: clear it and go without
        c->K64_alt = nullptr;
        return NB2_OK;
    }
    NB2_CUDA(c, cudaStreamCreateWithFlags(&c->zstream, cudaStreamNonBlocking));
    NB2_CUDA(c, cudaEventCreateWithFlags(&c->zev_free, cudaEventDisableTiming));
    NB2_CUDA(c, cudaEventCreateWithFlags(&c->zev_done, cudaEventDisableTiming));
    c->kalt_state = 1;
    return NB2_OK;
}

extern "C" {

int nb2_create(const nb2_mesh_desc* m, const nb2_material* mat, nb2_ctx** out) {
    if (!out) return NB2_E_INPUT;
    *out = nullptr;
    if (!m || !mat || !m->coordinates || !m->connectivity || m->num_nodes <= 0 ||
        m->num_elements <= 0 || (m->nodes_per_element != 8 && m->nodes_per_element != 4) ||
        mat->model < 0 || mat->model > 5 ||
        (mat->unit_sphere_points != 0 && mat->unit_sphere_points != 21 &&
         mat->unit_sphere_points != 33)) {
        g_create_error = "invalid mesh or material description";
        return NB2_E_INPUT;
    }
    for (long long i = 0; i < (long long)m->num_elements * m->nodes_per_element; ++i)
        if (m->connectivity[i] < 0 || m->connectivity[i] >= m->num_nodes) {
            g_create_error = "connectivity refers to a node outside the coordinate list";
            return NB2_E_INPUT;
        }
    if ((long long)m->num_elements * (m->nodes_per_element == 8 ? 8 : 1) >= (1ll << 31)) {
        g_create_error = "too many quadrature points for 32-bit indexing";
        return NB2_E_INPUT;
    }
    auto* c = new nb2_ctx();
    c->N = m->num_nodes;
    c->E = m->num_elements;
    c->npe = m->nodes_per_element;
    c->nq = c->npe == 8 ? 8 : 1;
    c->nqp = c->E * c->nq;
    c->n = 3 * c->N;
    c->mat = *mat;
    auto fail = [&](int st) {
        g_create_error = c->error;
        nb2_destroy(c);
        return st;
    };
    cudaError_t e = cudaGetDevice(&c->device);
    if (e != cudaSuccess) return fail(cuda_fail(c, e, "cudaGetDevice"));
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(c, e, "cudaStreamCreate"));
    c->own_stream = true;
    int st = NB2_OK;
    if ((st = dev_alloc(c, &c->X, 3ll * c->N))) return fail(st);
    if ((st = dev_alloc(c, &c->conn, (long long)c->E * c->npe))) return fail(st);
    e = cudaMemcpyAsync(c->X, m->coordinates, sizeof(double) * 3 * c->N, cudaMemcpyHostToDevice,
                        c->stream);
    if (e != cudaSuccess) return fail(cuda_fail(c, e, "upload coordinates"));
    e = cudaMemcpyAsync(c->conn, m->connectivity, sizeof(int) * (size_t)c->E * c->npe,
                        cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return fail(cuda_fail(c, e, "upload connectivity"));
    if ((st = build_pattern(c))) return fail(st);
    double** vecs[] = {&c->u, &c->u_old, &c->fint, &c->fext, &c->rhs, &c->du, &c->inc,
                       &c->cg_x, &c->cg_r, &c->cg_p, &c->cg_q, &c->cg_inv};
    for (double** v : vecs)
        if ((st = dev_alloc(c, v, (long long)c->n))) return fail(st);
    if ((st = dev_alloc(c, &c->mask, (long long)c->n))) return fail(st);
    if ((st = dev_alloc(c, &c->partials, (long long)reduction_blocks(c) * 8))) return fail(st);
    if ((st = dev_alloc(c, &c->cgs, 1ll))) return fail(st);
    if ((st = dev_alloc(c, &c->norms, 8ll))) return fail(st);
    if ((st = dev_alloc(c, &c->status, 1ll))) return fail(st);
    if (c->mat.model == NB2_SMALL_STRAIN_J2_PLASTICITY) {
        if ((st = dev_alloc(c, &c->ep, 6ll * c->nqp))) return fail(st);
        if ((st = dev_alloc(c, &c->epbar, (long long)c->nqp))) return fail(st);
        if ((st = dev_alloc(c, &c->ep_old, 6ll * c->nqp))) return fail(st);
        if ((st = dev_alloc(c, &c->epbar_old, (long long)c->nqp))) return fail(st);
    }
    e = cudaMallocHost(&c->h_cgs, sizeof(CgScalars));
    if (e != cudaSuccess) return fail(cuda_fail(c, e, "cudaMallocHost"));
    e = cudaMallocHost(&c->h_norms, 8 * sizeof(double));
    if (e != cudaSuccess) return fail(cuda_fail(c, e, "cudaMallocHost"));
    if ((st = reset_status(c))) return fail(st);
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(cuda_fail(c, e, "create"));
    *out = c;
    return NB2_OK;
}

int nb2_destroy(nb2_ctx* c) {
    if (!c) return NB2_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    release_graphs(c);
    void* ptrs[] = {c->X,      c->conn,   c->brp,    c->bcol,   c->slot,      c->K64,
                    c->K32,    c->u,      c->u_old,  c->fint,   c->fext,      c->rhs,
                    c->du,     c->inc,    c->mask,   c->Ge,     c->Ke,        c->ep,
                    c->epbar,  c->u_tan, c->Kcsr, c->mf_d, c->mf_c, c->mf_ye, c->nadj, c->nadj_ptr, c->nadj_pl,
                    c->ep_old, c->epbar_old, c->sig, c->dpar,   c->detF,      c->cg_x,
                    c->cg_r,   c->cg_p,   c->cg_q,   c->cg_inv, c->cg32_x,    c->cg32_r,
                    c->cg32_p, c->cg32_q, c->cg32_inv, c->partials, c->cgs,   c->norms,
                    c->status, c->corder, c->K64_alt};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->zev_free) cudaEventDestroy(c->zev_free);
    if (c->zev_done) cudaEventDestroy(c->zev_done);
    if (c->zstream) cudaStreamDestroy(c->zstream);
    if (c->h_cgs) cudaFreeHost(c->h_cgs);
    if (c->h_norms) cudaFreeHost(c->h_norms);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return NB2_OK;
}

int nb2_last_error(const nb2_ctx* c, char* buf, size_t size) {
    if (!buf || size == 0) return NB2_E_INPUT;
    const std::string& s = c ? c->error : g_create_error;
    std::snprintf(buf, size, "%s", s.c_str());
    return NB2_OK;
}

int nb2_set_stream(nb2_ctx* c, void* stream) {
    if (!c) return NB2_E_INPUT;
    cudaStreamSynchronize(c->stream);
    release_graphs(c);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    return NB2_OK;
}

int nb2_element_stiffness(nb2_ctx* c, int64_t element, double* Ke) {
    if (!c || !Ke || element < 0 || element >= c->E) return NB2_E_INPUT;
    const size_t nd = 3 * (size_t)c->npe;
    double* d = nullptr;
    NB2_CUDA(c, cudaMallocAsync(&d, sizeof(double) * nd * nd, c->stream));
    int st = launch_element_stiffness(c, element, d);
    if (st == NB2_OK) {
        NB2_CUDA(c, cudaMemcpyAsync(Ke, d, sizeof(double) * nd * nd, cudaMemcpyDeviceToHost,
                                    c->stream));
    }
    cudaFreeAsync(d, c->stream);
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return st;
}

int nb2_set_scatter_mode(nb2_ctx* c, int32_t mode) {
    if (!c || (mode != NB2_SCATTER_RED && mode != NB2_SCATTER_COLOURED)) return NB2_E_INPUT;
    c->scatter = mode;
    return NB2_OK;
}

int nb2_get_sizes(const nb2_ctx* c, int32_t* n, int64_t* nnz, int64_t* nb) {
    if (!c) return NB2_E_INPUT;
    if (n) *n = c->n;
    if (nnz) *nnz = c->nnz;
    if (nb) *nb = c->nnzb;
    return NB2_OK;
}

int nb2_launch_count(const nb2_ctx* c, int64_t* launches) {
    if (!c || !launches) return NB2_E_INPUT;
    *launches = c->launches;
    return NB2_OK;
}

int nb2_set_element_shear_modulus(nb2_ctx* c, const double* G) {
    if (!c || !G) return NB2_E_INPUT;
    if (!c->Ge) NB2_TRY(dev_alloc(c, &c->Ge, (long long)c->E));
    NB2_CUDA(c, cudaMemcpyAsync(c->Ge, G, sizeof(double) * c->E, cudaMemcpyHostToDevice, c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

int nb2_set_element_moduli(nb2_ctx* c, const double* K, const double* G) {
    if (!c || (!K && !G)) return NB2_E_INPUT;
    if (c->mat.model == NB2_SMALL_STRAIN_J2_PLASTICITY) {
        c->error = "per-element moduli are not supported for J2 plasticity";
        return NB2_E_INPUT;
    }
    if (G) NB2_TRY(nb2_set_element_shear_modulus(c, G));
    if (K) {
        if (!c->Ke) NB2_TRY(dev_alloc(c, &c->Ke, (long long)c->E));
        NB2_CUDA(c, cudaMemcpyAsync(c->Ke, K, sizeof(double) * c->E, cudaMemcpyHostToDevice,
                                    c->stream));
        NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return NB2_OK;
}

int nb2_export_pattern(nb2_ctx* c, int32_t* rowptr, int32_t* col) {
    if (!c || !rowptr || !col) return NB2_E_INPUT;
    long long pos = 0;
    rowptr[0] = 0;
    for (int a = 0; a < c->N; ++a) {
        const int b0 = c->h_brp[a], b1 = c->h_brp[a + 1];
        for (int r = 0; r < 3; ++r) {
            for (int k = b0; k < b1; ++k)
                for (int cc = 0; cc < 3; ++cc) col[pos++] = 3 * c->h_bcol[k] + cc;
            rowptr[3 * a + r + 1] = (int32_t)pos;
        }
    }
    return NB2_OK;
}

int nb2_set_displacement(nb2_ctx* c, const double* u) {
    if (!c || !u) return NB2_E_INPUT;
    NB2_CUDA(c, cudaMemcpyAsync(c->u, u, sizeof(double) * c->n, cudaMemcpyHostToDevice, c->stream));
    return NB2_OK;
}

int nb2_get_displacement(nb2_ctx* c, double* u) {
    if (!c || !u) return NB2_E_INPUT;
    NB2_CUDA(c, cudaMemcpyAsync(u, c->u, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

int nb2_update_internal_variables(nb2_ctx* c, const double* u, double) {
    if (!c || !u) return NB2_E_INPUT;
    NB2_TRY(ensure_split_buffers(c));
    NB2_TRY(nb2_set_displacement(c, u));
    NB2_TRY(reset_status(c));
    NB2_TRY(launch_element_kernel(c, MODE_CONSTITUTIVE | MODE_STORE, NB2_FP64));
    return read_status(c);
}

int nb2_assemble(nb2_ctx* c, double* K, double* f) {
    if (!c) return NB2_E_INPUT;
    if (!c->sig) {
        c->error = "nb2_assemble needs a prior nb2_update_internal_variables";
        return NB2_E_INPUT;
    }
    NB2_TRY(ensure_k64(c));
    NB2_TRY(launch_element_kernel(c, MODE_STIFFNESS | MODE_FORCE, NB2_FP64));
    return nb2_download_system(c, K, f);
}

int nb2_download_system(nb2_ctx* c, double* K, double* f) {
    if (!c) return NB2_E_INPUT;
    if (K) {
        if (!c->K64) return NB2_E_INPUT;
        // CSR staging buffer kept for the context's lifetime (one 8 nnz-byte allocation, not one
        // per call); the copy runs at DMA speed when the caller's buffer is page-locked
        if (!c->Kcsr) NB2_CUDA(c, cudaMalloc(&c->Kcsr, sizeof(double) * c->nnz));
        NB2_TRY(export_csr_values(c, c->K64, c->Kcsr));
        NB2_CUDA(c, cudaMemcpyAsync(K, c->Kcsr, sizeof(double) * c->nnz, cudaMemcpyDeviceToHost,
                                    c->stream));
    }
    if (f)
        NB2_CUDA(c, cudaMemcpyAsync(f, c->fint, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                                    c->stream));
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

int nb2_save_internal_variables(nb2_ctx* c, int32_t converged) {
    if (!c) return NB2_E_INPUT;
    if (c->ep) {
        const size_t b6 = sizeof(double) * 6 * (size_t)c->nqp, b1 = sizeof(double) * c->nqp;
        if (converged) {
            NB2_CUDA(c, cudaMemcpyAsync(c->ep_old, c->ep, b6, cudaMemcpyDeviceToDevice, c->stream));
            NB2_CUDA(c, cudaMemcpyAsync(c->epbar_old, c->epbar, b1, cudaMemcpyDeviceToDevice,
                                        c->stream));
        } else {
            NB2_CUDA(c, cudaMemcpyAsync(c->ep, c->ep_old, b6, cudaMemcpyDeviceToDevice, c->stream));
            NB2_CUDA(c, cudaMemcpyAsync(c->epbar, c->epbar_old, b1, cudaMemcpyDeviceToDevice,
                                        c->stream));
        }
    }
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

int nb2_get_quadrature_values(nb2_ctx* c, int32_t which, double* out) {
    if (!c || !out) return NB2_E_INPUT;
    const long long nqp = c->nqp;
    double* tmp = nullptr;
    if (which == 0 || which == 2) {
        const double* src = which == 0 ? c->sig : c->ep;
        if (!src) {
            if (which == 2) {
                std::memset(out, 0, sizeof(double) * 9 * nqp);
                return NB2_OK;
            }
            return NB2_E_INPUT;
        }
        NB2_CUDA(c, cudaMallocAsync(&tmp, sizeof(double) * 9 * nqp, c->stream));
        k_sym6_to_9<<<(unsigned)((nqp + 255) / 256), 256, 0, c->stream>>>(nqp, src, tmp);
        c->launches++;
        NB2_CUDA(c, cudaMemcpyAsync(out, tmp, sizeof(double) * 9 * nqp, cudaMemcpyDeviceToHost,
                                    c->stream));
        NB2_CUDA(c, cudaFreeAsync(tmp, c->stream));
    } else if (which == 1 || which == 3) {
        const double* src = which == 1 ? c->detF : c->epbar;
        if (!src) {
            if (which == 3) {
                std::memset(out, 0, sizeof(double) * nqp);
                return NB2_OK;
            }
            return NB2_E_INPUT;
        }
        NB2_CUDA(c, cudaMemcpyAsync(out, src, sizeof(double) * nqp, cudaMemcpyDeviceToHost,
                                    c->stream));
    } else {
        return NB2_E_INPUT;
    }
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

int nb2_apply_dirichlet(nb2_ctx* c, const int32_t* dofs, int32_t nd, double* K, double* b) {
    if (!c || (!dofs && nd > 0) || !K || !b) return NB2_E_INPUT;
    // static_matrix::enforce_dirichlet_conditions on the neon CSR layout
    std::vector<long long> rowptr(c->n + 1);
    rowptr[0] = 0;
    for (int a = 0; a < c->N; ++a) {
        const long long deg = c->h_brp[a + 1] - c->h_brp[a];
        for (int r = 0; r < 3; ++r) rowptr[3 * a + r + 1] = rowptr[3 * a + r] + 3 * deg;
    }
    auto find = [&](int row, int col) -> long long {
        const int a = row / 3;
        const int* s = c->h_bcol.data() + c->h_brp[a];
        const int* e = c->h_bcol.data() + c->h_brp[a + 1];
        const int* p = std::lower_bound(s, e, col / 3);
        if (p == e || *p != col / 3) return -1;
        return rowptr[row] + 3 * (p - s) + col % 3;
    };
    for (int i = 0; i < nd; ++i) {
        const int d = dofs[i];
        if (d < 0 || d >= c->n) return NB2_E_INPUT;
        const long long pd = find(d, d);
        const double diag = K[pd];
        b[d] = 0.0;
        const int a = d / 3;
        for (int k = c->h_brp[a]; k < c->h_brp[a + 1]; ++k)
            for (int cc = 0; cc < 3; ++cc) {
                const int col = 3 * c->h_bcol[k] + cc;
                K[find(d, col)] = 0.0;
                K[find(col, d)] = 0.0;
            }
        K[pd] = diag;
    }
    return NB2_OK;
}

int nb2_pcg_solve(int32_t n, const int32_t* rowptr, const int32_t* col, const double* values,
                  const double* b, double* x, double tol, int32_t maxit, int32_t* iterations,
                  double* error) {
    if (n <= 0 || !rowptr || !col || !values || !b || !x || maxit <= 0) return NB2_E_INPUT;
    // the device kernels index x[col[k]] and rows rowptr[i]..rowptr[i+1]: validate first
    if (rowptr[0] != 0) return NB2_E_INPUT;
    for (int i = 0; i < n; ++i)
        if (rowptr[i + 1] < rowptr[i]) return NB2_E_INPUT;
    for (long long k = 0; k < rowptr[n]; ++k)
        if (col[k] < 0 || col[k] >= n) return NB2_E_INPUT;
    int it = 0;
    double err = 0;
    std::string msg;
    int st = pcg_csr_host(n, rowptr, col, values, b, x, tol, maxit, &it, &err, &msg);
    if (iterations) *iterations = it;
    if (error) *error = err;
    if (st == NB2_OK) {
        for (int i = 0; i < n; ++i)
            if (std::isnan(x[i])) return NB2_E_NAN;
    }
    return st;
}

int nb2_update_assemble_device(nb2_ctx* c, int32_t precision) {
    if (!c) return NB2_E_INPUT;
    if (precision == NB2_FP64)
        NB2_TRY(ensure_k64(c));
    else
        NB2_TRY(ensure_k32(c));
    return launch_element_kernel(c, MODE_CONSTITUTIVE | MODE_STIFFNESS | MODE_FORCE, precision);
}

int nb2_synchronize(nb2_ctx* c) {
    if (!c) return NB2_E_INPUT;
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

int nb2_apply_tangent_fp32(nb2_ctx* c, const double* v, double* y) {
    if (!c || !v || !y) return NB2_E_INPUT;
    if (!c->dpar) {
        c->error = "nb2_apply_tangent_fp32 needs a prior nb2_update_internal_variables";
        return NB2_E_INPUT;
    }
    double *dv = nullptr, *dy = nullptr;
    NB2_CUDA(c, cudaMallocAsync(&dv, sizeof(double) * c->n, c->stream));
    NB2_CUDA(c, cudaMallocAsync(&dy, sizeof(double) * c->n, c->stream));
    NB2_CUDA(c, cudaMemcpyAsync(dv, v, sizeof(double) * c->n, cudaMemcpyHostToDevice, c->stream));
    int st = mf_apply(c, dv, dy);
    if (st == NB2_OK)
        NB2_CUDA(c, cudaMemcpyAsync(y, dy, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                                    c->stream));
    cudaFreeAsync(dv, c->stream);
    cudaFreeAsync(dy, c->stream);
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return st;
}

int nb2_apply_tangent(nb2_ctx* c, const double* v, double* y) {
    if (!c || !v || !y) return NB2_E_INPUT;
    if (!c->dpar) {
        c->error = "nb2_apply_tangent needs a prior nb2_update_internal_variables";
        return NB2_E_INPUT;
    }
    double *dv = nullptr, *dy = nullptr;
    NB2_CUDA(c, cudaMallocAsync(&dv, sizeof(double) * c->n, c->stream));
    NB2_CUDA(c, cudaMallocAsync(&dy, sizeof(double) * c->n, c->stream));
    NB2_CUDA(c, cudaMemcpyAsync(dv, v, sizeof(double) * c->n, cudaMemcpyHostToDevice, c->stream));
    int st = launch_apply(c, dv, dy);
    if (st == NB2_OK)
        NB2_CUDA(c, cudaMemcpyAsync(y, dy, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                                    c->stream));
    cudaFreeAsync(dv, c->stream);
    cudaFreeAsync(dy, c->stream);
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return st;
}

int nb2_set_dirichlet_mask(nb2_ctx* c, const int32_t* dofs, int32_t nd) {
    if (!c || (nd > 0 && !dofs)) return NB2_E_INPUT;
    for (int i = 0; i < nd; ++i)
        if (dofs[i] < 0 || dofs[i] >= c->n) return NB2_E_INPUT;
    NB2_CUDA(c, cudaMemsetAsync(c->mask, 0, c->n, c->stream));
    if (nd > 0) {
        int* d = nullptr;
        NB2_CUDA(c, cudaMallocAsync(&d, sizeof(int) * nd, c->stream));
        NB2_CUDA(c, cudaMemcpyAsync(d, dofs, sizeof(int) * nd, cudaMemcpyHostToDevice, c->stream));
        k_scatter_mask<<<(nd + 255) / 256, 256, 0, c->stream>>>(nd, d, c->mask);
        c->launches++;
        NB2_CUDA(c, cudaFreeAsync(d, c->stream));
    }
    NB2_CUDA(c, cudaStreamSynchronize(c->stream));
    return NB2_OK;
}

int nb2_solve_device(nb2_ctx* c, int32_t precision, double tol, int32_t maxit, int32_t* iterations,
                     double* error) {
    if (!c || maxit <= 0) return NB2_E_INPUT;
    if ((precision == NB2_FP64 && !c->K64) || (precision != NB2_FP64 && !c->K32)) {
        c->error = "nb2_solve_device needs an assembled K of that precision";
        return NB2_E_INPUT;
    }
    NB2_CUDA(c, cudaMemcpyAsync(c->rhs, c->fint, sizeof(double) * c->n, cudaMemcpyDeviceToDevice,
                                c->stream));
    k_zero_masked<<<grid_for(c->n), 256, 0, c->stream>>>(c->n, c->mask, c->rhs);
    c->launches++;
    int it = 0;
    double err = 0;
    int st = precision == NB2_FP64
                 ? pcg_device_fp64(c, c->rhs, c->du, tol, maxit, true, &it, &err, true)
                 : pcg_device_fp32(c, c->rhs, c->du, tol, maxit, &it, &err, true);
    if (iterations) *iterations = it;
    if (error) *error = err;
    if (st == NB2_E_CG_MAXIT && tol == 0.0) st = NB2_OK;  // fixed-count timing run
    return st;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Defect correction for K_outer out = rhs (masked rows): restarted inner PCG solves on an
// approximate operator (inner: NB2_MIXED = FP32 K32, NB2_FP64 = K64) to the relative tolerance
// inner_tol, each correcting the residual rhs - K_outer out formed in FP64 with K_outer = the
// stored tangent applied matrix-free, or (exact) the forward-mode product (d f_int/du) v.  out
// converges to the solution of the outer system to the relative tolerance `tol`.  rlin, corr,
// yvec: n-vector work space.  The Newton path's mixed solve (same operator inside and out) uses
// the reliable-update PCG instead, which keeps its Krylov space across residual replacements.
// ---------------------------------------------------------------------------------------
static int solve_defect_corrected(nb2_ctx* c, const double* rhs, double* out, double tol,
                                  double inner_tol, int maxit, bool graphs, double* rlin,
                                  double* corr, double* yvec, int* iterations, int inner,
                                  bool exact);

static int solve_mixed_system(nb2_ctx* c, const double* rhs, double* out, double tol,
                              double inner_tol, int maxit, bool graphs, double* rlin,
                              double* corr, double* yvec, int* iterations) {
    (void)rlin;
    (void)corr;
    return pcg_reliable_mixed(c, rhs, out, tol, inner_tol, maxit, yvec, iterations, graphs,
                              true);
}

static int solve_defect_corrected(nb2_ctx* c, const double* rhs, double* out, double tol,
                                  double inner_tol, int maxit, bool graphs, double* rlin,
                                  double* corr, double* yvec, int* iterations, int inner,
                                  bool exact) {
    const unsigned g = grid_for(c->n);
    const double b2 = device_dot_sync(c, rhs, rhs, c->n);
    const double thr = std::max(tol * tol * b2, 2.2250738585072014e-308);
    NB2_CUDA(c, cudaMemsetAsync(out, 0, sizeof(double) * c->n, c->stream));
    NB2_CUDA(c, cudaMemcpyAsync(rlin, rhs, sizeof(double) * c->n, cudaMemcpyDeviceToDevice,
                                c->stream));
    int total = 0;
    double r2 = b2;
    for (int ref = 0; ref < 30 && r2 >= thr && b2 > 0; ++ref) {
        int it = 0;
        double err = 0;
        int st = inner == NB2_FP64
                     ? pcg_device_fp64(c, rlin, corr, inner_tol, std::max(1, maxit - total), true,
                                       &it, &err, graphs)
                     : pcg_device_fp32(c, rlin, corr, inner_tol, std::max(1, maxit - total), &it,
                                       &err, graphs);
        total += it;
        if (st && st != NB2_E_CG_MAXIT) {
            *iterations = total;
            return st;
        }
        k_axpy<<<g, 256, 0, c->stream>>>(c->n, 1.0, corr, out);
        if (exact)
            NB2_TRY(launch_force_jvp(c, out, yvec));
        else
            NB2_TRY(launch_apply(c, out, yvec));
        k_sub<<<g, 256, 0, c->stream>>>(c->n, rhs, yvec, rlin);
        k_zero_masked<<<g, 256, 0, c->stream>>>(c->n, c->mask, rlin);
        c->launches += 3;
        r2 = device_dot_sync(c, rlin, rlin, c->n);
        if (std::getenv("NB2_DEBUG"))
            std::fprintf(stderr, "[nb2] defect correction %d: inner its %d (status %d) |r|^2 %.6e "
                         "b^2 %.6e threshold %.6e\n", ref, it, st, r2, b2, thr);
        if (total >= maxit) break;
    }
    *iterations = total;
    if (!std::isfinite(r2)) return NB2_E_NAN;
    if (r2 >= thr && b2 > 0) return NB2_E_CG_MAXIT;
    return NB2_OK;
}

// Adjoint gradient of J(u) with respect to the per-element shear modulus of the microsphere
// model at the context's displacement (the converged state of the last nb2_static_solve, whose
// Dirichlet mask is still set).  Transpose solve on the tangent (K is symmetric), then
// dJ/dG_e = -lambda^T df_int/dG_e.
extern "C" int nb2_adjoint_shear_gradient(nb2_ctx* c, const double* dJdu, int32_t precision,
                                          double tol, int32_t maxit, double* dJdG,
                                          int32_t* iterations) {
    if (!c || !dJdu || !dJdG || maxit <= 0) return NB2_E_INPUT;
    if (c->mat.model != NB2_GAUSSIAN_AFFINE_MICROSPHERE &&
        c->mat.model != NB2_LANGEVIN_AFFINE_MICROSPHERE) {
        c->error = "the shear-modulus adjoint is defined for the affine microsphere models";
        return NB2_E_INPUT;
    }
    if (!c->Ge) {  // uniform field = the material modulus
        std::vector<double> g(c->E, c->mat.shear_modulus);
        NB2_TRY(nb2_set_element_shear_modulus(c, g.data()));
    }
    const bool mixed = precision == NB2_MIXED;
    NB2_TRY(mixed ? ensure_k32(c) : ensure_k64(c));
    if (mixed) NB2_TRY(ensure_split_buffers(c));
    NB2_CUDA(c, cudaMemcpyAsync(c->rhs, dJdu, sizeof(double) * c->n, cudaMemcpyHostToDevice,
                                c->stream));
    k_zero_masked<<<grid_for(c->n), 256, 0, c->stream>>>(c->n, c->mask, c->rhs);
    c->launches++;
    // tangent at the converged displacement (the microsphere has no history: no state change)
    NB2_TRY(reset_status(c));
    int mode = MODE_CONSTITUTIVE | MODE_STIFFNESS | MODE_FORCE | (mixed ? MODE_STORE : 0);
    NB2_TRY(launch_element_kernel(c, mode, mixed ? NB2_MIXED : NB2_FP64));
    NB2_TRY(read_status(c));
    int it = 0;
    int st;
    double *rl = nullptr, *co = nullptr, *yv = nullptr, *grad = nullptr;
    NB2_CUDA(c, cudaMalloc(&grad, sizeof(double) * c->E));
    NB2_CUDA(c, cudaMalloc(&rl, sizeof(double) * c->n));
    NB2_CUDA(c, cudaMalloc(&co, sizeof(double) * c->n));
    NB2_CUDA(c, cudaMalloc(&yv, sizeof(double) * c->n));
    // neon's assembled tangent is not the exact derivative of f_int: solve the exact system by
    // defect correction, the assembled K (FP64, or FP32 for the mixed adjoint) as inner solver
    // and the forward-mode product (d f_int/du) lambda as residual
    st = solve_defect_corrected(c, c->rhs, c->du, tol, mixed ? 1e-4 : 1e-6, maxit, true, rl, co,
                                yv, &it, mixed ? NB2_MIXED : NB2_FP64, true);
    if (iterations) *iterations = it;
    if (st == NB2_OK) st = launch_adjoint_shear(c, c->du, grad);
    if (st == NB2_OK) {
        cudaMemcpyAsync(dJdG, grad, sizeof(double) * c->E, cudaMemcpyDeviceToHost, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) st = NB2_E_CUDA;
    }
    for (double* p : {rl, co, yv, grad})
        if (p) cudaFree(p);
    return st;
}

// ---------------------------------------------------------------------------------------
// static_matrix (src/assembler/mechanics/static_matrix.hpp:29-467) over device state
// ---------------------------------------------------------------------------------------
namespace {

struct DeviceTable {
    TimeTable table;
    int* dofs = nullptr;
    double* weights = nullptr;
    int count = 0;
};

struct Newton {
    nb2_ctx* c;
    nb2_solver_options o;
    std::vector<DeviceTable> dirichlet, forces;
    AdaptiveTimeStep load;
    bool use_relative_norm = true;
    double norm_initial_residual = 1.0, displacement_norm = 0.0, force_norm = 0.0;
    std::vector<nb2_newton_log> log;
    long long newton_iterations = 0, cg_iterations = 0;
    double t_elem = 0, t_solve = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int last_cg = 0;

    ~Newton() {
        for (auto* v : {&dirichlet, &forces})
            for (auto& t : *v) {
                if (t.dofs) cudaFree(t.dofs);
                if (t.weights) cudaFree(t.weights);
            }
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (double* p : {rlin, corr, yvec})
            if (p) cudaFree(p);
    }

    int upload(const nb2_dof_table* in, int count, std::vector<DeviceTable>& out, bool weighted) {
        for (int i = 0; i < count; ++i) {
            DeviceTable d;
            const nb2_dof_table& t = in[i];
            if (t.num_points < 1 || t.num_dofs < 0 || (t.num_dofs > 0 && !t.dofs) || !t.times ||
                !t.values)
                return NB2_E_INPUT;
            for (int k = 0; k < t.num_dofs; ++k)
                if (t.dofs[k] < 0 || t.dofs[k] >= c->n) return NB2_E_INPUT;
            d.table.t.assign(t.times, t.times + t.num_points);
            d.table.v.assign(t.values, t.values + t.num_points);
            d.count = t.num_dofs;
            NB2_CUDA(c, cudaMalloc(&d.dofs, sizeof(int) * std::max(1, t.num_dofs)));
            NB2_CUDA(c, cudaMemcpyAsync(d.dofs, t.dofs, sizeof(int) * t.num_dofs,
                                        cudaMemcpyHostToDevice, c->stream));
            if (weighted && t.weights) {
                NB2_CUDA(c, cudaMalloc(&d.weights, sizeof(double) * std::max(1, t.num_dofs)));
                NB2_CUDA(c, cudaMemcpyAsync(d.weights, t.weights, sizeof(double) * t.num_dofs,
                                            cudaMemcpyHostToDevice, c->stream));
            }
            out.push_back(std::move(d));
        }
        return NB2_OK;
    }

    void time_begin() { cudaEventRecord(ev0, c->stream); }
    double time_end() {
        cudaEventRecord(ev1, c->stream);
        cudaEventSynchronize(ev1);
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        return ms * 1e-3;
    }

    unsigned grid() const { return grid_for(c->n); }

    double *rlin = nullptr, *corr = nullptr, *yvec = nullptr;  // mixed defect correction

    int alloc_mixed() {
        NB2_CUDA(c, cudaMalloc(&rlin, sizeof(double) * c->n));
        NB2_CUDA(c, cudaMalloc(&corr, sizeof(double) * c->n));
        NB2_CUDA(c, cudaMalloc(&yvec, sizeof(double) * c->n));
        return NB2_OK;
    }

    bool mixed() const { return o.precision == NB2_MIXED; }

    // update (+ assemble) at the context displacement; the mixed path also stores the FP64
    // tangent coefficients for its matrix-free defect residual
    int element_pass(bool assemble) {
        NB2_TRY(reset_status(c));
        time_begin();
        // mixed: no assembled K at all -- the stored FP64 tangent feeds the lifting, the FP64
        // residual replacements and the FP32 matrix-free operator of the PCG.  The update without
        // assembly (at a converged displacement, or at the start of a load attempt) stores its
        // point outputs, which the nodal averages of the file output read.
        int mode = MODE_CONSTITUTIVE | MODE_FORCE;
        if (assemble)
            mode |= mixed() ? MODE_STORE : MODE_STIFFNESS;
        else
            mode |= MODE_STORE;
        NB2_TRY(launch_element_kernel(c, mode, NB2_FP64));
        t_elem += time_end();
        return read_status(c);
    }

    int compute_external_force() {
        NB2_CUDA(c, cudaMemsetAsync(c->fext, 0, sizeof(double) * c->n, c->stream));
        const double t = load.step_time();
        for (auto& f : forces) {
            if (f.count == 0) continue;
            k_scatter_add_weighted<<<(f.count + 255) / 256, 256, 0, c->stream>>>(
                f.count, f.dofs, f.weights, f.table.value(t), c->fext);
            c->launches++;
        }
        return NB2_OK;
    }

    int set_mask() {
        NB2_CUDA(c, cudaMemsetAsync(c->mask, 0, c->n, c->stream));
        for (auto& d : dirichlet) {
            if (!d.table.active(load.step_time()) || d.count == 0) continue;
            k_scatter_mask<<<(d.count + 255) / 256, 256, 0, c->stream>>>(d.count, d.dofs, c->mask);
            c->launches++;
        }
        return NB2_OK;
    }

    // static_matrix::apply_displacement_boundaries (:322-351)
    int apply_displacement_boundaries() {
        NB2_CUDA(c, cudaMemsetAsync(c->inc, 0, sizeof(double) * c->n, c->stream));
        for (auto& d : dirichlet) {
            if (!d.table.active(load.step_time()) || d.count == 0) continue;
            const double du = d.table.value(load.step_time()) -
                              d.table.value(load.last_converged_time);
            k_scatter_set<<<(d.count + 255) / 256, 256, 0, c->stream>>>(d.count, d.dofs, du, c->inc);
            c->launches++;
        }
        double* tmp = c->cg_q;  // free until the solve
        if (mixed())
            NB2_TRY(launch_apply(c, c->inc, tmp));  // FP64 tangent, matrix-free
        else
            bsr_spmv_fp64(c, c->inc, tmp, false);
        k_axpy<<<grid(), 256, 0, c->stream>>>(c->n, -1.0, tmp, c->rhs);
        k_axpy<<<grid(), 256, 0, c->stream>>>(c->n, 1.0, c->inc, c->u);
        c->launches += 2;
        return NB2_OK;
    }

    void update_relative_norms() {
        const double* nv = c->h_norms;  // du, u, rhs, fext, fint
        if (use_relative_norm && !is_approx(nv[1], 0.0, 1.0) &&
            !is_approx(std::max(nv[3], nv[4]), 0.0, 1.0)) {
            displacement_norm = nv[0] / nv[1];
            force_norm = nv[2] / std::max(norm_initial_residual, std::max(nv[3], nv[4]));
        } else {
            displacement_norm = nv[0];
            force_norm = nv[2];
        }
    }

    // Mixed precision: FP64 defect correction around FP32 inner PCG solves.  The defect
    // rlin = rhs - K du uses the FP64 tangent (matrix-free), so du converges to the solution of
    // the same FP64 system as the FP64 path, to the same relative tolerance.
    int solve_mixed(int* iterations) {
        return solve_mixed_system(c, c->rhs, c->du, o.cg_tolerance, o.mixed_inner_tolerance,
                                  o.cg_maximum_iterations, o.use_graphs != 0, rlin, corr, yvec,
                                  iterations);
    }

    int solve_linear() {
        int it = 0;
        double err = 0;
        time_begin();
        int st;
        if (mixed())
            st = solve_mixed(&it);
        else
            st = pcg_device_fp64(c, c->rhs, c->du, o.cg_tolerance, o.cg_maximum_iterations, true,
                                 &it, &err, o.use_graphs != 0);
        t_solve += time_end();
        last_cg = it;
        cg_iterations += it;
        if (st == NB2_E_CG_MAXIT) c->error = "Conjugate gradient solver maximum iterations reached";
        if (st == NB2_E_NAN || st == NB2_E_CG_BREAKDOWN) c->error = "Floating point error reported";
        return st;
    }

    // perform_equilibrium_iterations (:402-467); >0 recoverable error, <0 fatal
    int equilibrium() {
        NB2_CUDA(c, cudaMemcpyAsync(c->u, c->u_old, sizeof(double) * c->n, cudaMemcpyDeviceToDevice,
                                    c->stream));
        NB2_TRY(set_mask());
        // mesh.update_internal_variables(u_old) fused with the first assembly
        int st = element_pass(true);
        if (st) return st;
        int k = 0;
        while (k < o.linear_iterations) {
            k_sub<<<grid(), 256, 0, c->stream>>>(c->n, c->fext, c->fint, c->rhs);
            c->launches++;
            if (k == 0) {
                NB2_TRY(apply_displacement_boundaries());
                NB2_TRY(compute_norms(c));
                norm_initial_residual = c->h_norms[2];
            }
            k_zero_masked<<<grid(), 256, 0, c->stream>>>(c->n, c->mask, c->rhs);
            c->launches++;
            st = solve_linear();
            if (st) return st;
            k_axpy<<<grid(), 256, 0, c->stream>>>(c->n, 1.0, c->du, c->u);
            c->launches++;
            NB2_TRY(compute_norms(c));
            update_relative_norms();
            ++newton_iterations;
            log.push_back({load.step_time(), k, last_cg, displacement_norm, force_norm});
            const bool converged =
                displacement_norm <= o.displacement_tolerance && force_norm <= o.residual_tolerance;
            // mesh.update_internal_variables(u_{k+1}); the next assembly is fused into it
            st = element_pass(!converged);
            if (st) return st;
            if (converged) break;
            ++k;
        }
        if (k == o.linear_iterations) {
            c->error = "Reached Newton-Raphson iteration limit";
            return NB2_E_NEWTON_MAXIT;
        }
        NB2_CUDA(c, cudaMemcpyAsync(c->u_old, c->u, sizeof(double) * c->n, cudaMemcpyDeviceToDevice,
                                    c->stream));
        if (!load.update(true)) return -NB2_E_CUTBACK_LIMIT;
        NB2_TRY(nb2_save_internal_variables(c, 1));
        return NB2_OK;
    }

    // solve (:145-187) with the cutback recursion as a loop
    int solve() {
        NB2_CUDA(c, cudaMemsetAsync(c->u, 0, sizeof(double) * c->n, c->stream));
        NB2_CUDA(c, cudaMemsetAsync(c->u_old, 0, sizeof(double) * c->n, c->stream));
        for (;;) {
            int st = element_pass(false);
            bool failed = st != NB2_OK;
            if (st < 0 || st == NB2_E_CUDA || st == NB2_E_INPUT) return st < 0 ? -st : st;
            while (!failed && !load.is_applied) {
                NB2_TRY(compute_external_force());
                st = equilibrium();
                if (st < 0) return -st;
                if (st == NB2_E_CUDA || st == NB2_E_INPUT || st == NB2_E_TIMEOUT) return st;
                if (st != NB2_OK) failed = true;
            }
            if (!failed) return NB2_OK;
            if (!load.update(false)) {
                c->error = "Too many reductions.  Convergence not judged likely";
                return NB2_E_CUTBACK_LIMIT;
            }
            NB2_TRY(nb2_save_internal_variables(c, 0));
            NB2_CUDA(c, cudaMemcpyAsync(c->u, c->u_old, sizeof(double) * c->n,
                                        cudaMemcpyDeviceToDevice, c->stream));
        }
    }
};

}  // namespace

extern "C" int nb2_static_solve(nb2_ctx* c, const nb2_solver_options* options,
                                const nb2_dof_table* dirichlet, int32_t num_dirichlet,
                                const nb2_dof_table* nodal_forces, int32_t num_nodal_forces,
                                double* u_out, nb2_solve_report* report, nb2_newton_log* log,
                                int32_t max_log) {
    if (!c || !options || (num_dirichlet > 0 && !dirichlet) ||
        (num_nodal_forces > 0 && !nodal_forces))
        return NB2_E_INPUT;
    Newton nw;
    nw.c = c;
    nw.o = *options;
    if (nw.o.linear_iterations <= 0 || nw.o.cg_maximum_iterations <= 0) return NB2_E_INPUT;
    // the context's solver buffers (kept for later solves) are set up before the clock of the
    // report starts.  The mixed path assembles no K: its PCG runs on the FP32 matrix-free
    // operator, so it needs the FP32 vectors and that operator's buffers, not K32
    NB2_TRY(ensure_split_buffers(c));
    if (nw.o.precision == NB2_MIXED) {
        NB2_TRY(ensure_cg32(c));
        NB2_TRY(ensure_mf(c));
        NB2_TRY(nw.alloc_mixed());
        if (!(nw.o.mixed_inner_tolerance > 0)) nw.o.mixed_inner_tolerance = 1e-4;
    } else {
        NB2_TRY(ensure_k64(c));
        // the second K buffer the element passes zero in the background
        if (!c->e_inst) NB2_TRY(ensure_k64_alt(c));
    }
    // the element colouring of the Newton driver's (bit-reproducible) hex8 element passes
    if (c->npe == 8 && !c->e_inst) NB2_TRY(ensure_colouring(c));
    auto t0 = std::chrono::steady_clock::now();
    nw.use_relative_norm = options->absolute_tolerance == 0;
    NB2_CUDA(c, cudaEventCreate(&nw.ev0));
    NB2_CUDA(c, cudaEventCreate(&nw.ev1));
    NB2_TRY(nw.upload(dirichlet, num_dirichlet, nw.dirichlet, false));
    NB2_TRY(nw.upload(nodal_forces, num_nodal_forces, nw.forces, true));
    std::vector<double> history;
    for (auto* v : {&nw.dirichlet, &nw.forces})
        for (auto& t : *v) history.insert(history.end(), t.table.t.begin(), t.table.t.end());
    std::sort(history.begin(), history.end());
    history.erase(std::unique(history.begin(), history.end()), history.end());
    if (history.empty()) history = {0.0, options->period};
    nw.load.init(options->period, options->initial_increment, options->minimum_increment,
                 options->maximum_increment, options->adaptive != 0, history);
    c->error.clear();
    c->newton_scatter = true;  // bit-reproducible Newton: coloured element passes
    int st = nw.solve();
    c->newton_scatter = false;
    if (u_out) {
        cudaMemcpyAsync(u_out, c->u, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream);
        cudaStreamSynchronize(c->stream);
    }
    if (report) {
        report->status = st;
        report->load_steps = nw.load.successful_increments;
        report->newton_iterations = nw.newton_iterations;
        report->cg_iterations = nw.cg_iterations;
        report->seconds_total =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        report->seconds_update_assembly = nw.t_elem;
        report->seconds_solve = nw.t_solve;
        std::snprintf(report->message, sizeof report->message, "%s", c->error.c_str());
    }
    if (log)
        for (int i = 0; i < (int)nw.log.size() && i < max_log; ++i) log[i] = nw.log[i];
    return st;
}
