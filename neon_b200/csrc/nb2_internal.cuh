// nb2_internal.cuh -- context layout and device helpers shared by the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/neon_b200.h"

namespace nb2 {

// ---------------------------------------------------------------------------------------
// Device layout
//
//   nodes        X[N][3], u[N][3]  (node-major: DOF 3*node + k, gathers read 24 B per node)
//   elements     conn[E][npe]      (element-major: a group of lanes reads one element's row)
//   block pattern brp[N+1], bcol[nnzb]  (3x3 node blocks; CSR of neon = this pattern expanded)
//   values       K[nnzb][9]        (row-major 3x3 block, FP64 or FP32)
//   slot map     slot[E][npe*npe]  (block index of element block (a,b))
//   qp state     SoA: ep[6][nqp], epbar[nqp] (current) and their committed copies
//   qp outputs   sig[6][nqp], dpar[rows][nqp], detF[nqp] (only for the split update/assemble
//                path); dpar rows: lam', mu', b, then the J2 flow direction N (6) or, for the
//                Langevin and non-affine microsphere, the anisotropic tangent (21, packed
//                upper triangle)
// ---------------------------------------------------------------------------------------

// MODEL_MS: Gaussian affine microsphere, MODEL_ML: Langevin affine microsphere,
// MODEL_MN: non-affine microsphere
enum : int { MODEL_LE = 0, MODEL_NH = 1, MODEL_J2 = 2, MODEL_MS = 3, MODEL_ML = 4, MODEL_MN = 5 };

// models whose tangent carries a general anisotropic part Da (packed 6x6) besides lam', mu'
__host__ __device__ constexpr bool model_aniso(int model) {
    return model == MODEL_ML || model == MODEL_MN;
}

// rows of dpar for a model
inline int dpar_rows(int model) { return model_aniso(model) ? 3 + 21 : 9; }

// Packed index of the symmetric 6x6 (kinetic Voigt 11 22 33 23 13 12) entry (v, w): the upper
// triangle row by row.
__host__ __device__ constexpr int sym6(int v, int w) {
    return v <= w ? v * 6 - v * (v - 1) / 2 + (w - v) : w * 6 - w * (w - 1) / 2 + (v - w);
}

// element-kernel mode bits
enum : int {
    MODE_CONSTITUTIVE = 1,  // compute the constitutive update from u (else load stored outputs)
    MODE_STIFFNESS = 2,     // accumulate + scatter the tangent stiffness
    MODE_FORCE = 4,         // accumulate + scatter the internal force
    MODE_STORE = 8,         // store stress / tangent coefficients / det F per quadrature point
};

struct DeviceStatus {
    unsigned int flags;                // bit (status code - 1)
    unsigned int negdet_count;
    unsigned long long negdet_first;   // (qp index << 32) | float bits of det F
};

struct ElementArgs {
    const double* X;
    const double* u;
    const int* conn;
    const int* slot;
    int E;
    int nqp;
    double K, G, lambda, sigma_y, H_iso;
    double Nseg;       // segments per chain (Langevin and non-affine microsphere)
    double p_na;       // non-affine stretch parameter
    int sph0, nsph;    // unit-sphere rule of the microsphere models: first point, count
    const double* Ge;  // per-element shear modulus (or null)
    const double* Ke;  // per-element bulk modulus (or null)
    double* ep;      // [6][nqp]
    double* epbar;   // [nqp]
    double* K64;     // [nnzb][9]
    float* K32;
    double* fint;    // [3N]
    double* sig;     // [6][nqp]
    double* dpar;    // [dpar_rows(model)][nqp]
    double* detF;    // [nqp]
    DeviceStatus* status;
    // batched instances (all null outside a batched solve): element -> instance, the instances
    // whose elements this pass computes, per-instance status flags
    const int* e_inst;
    const int* inst_on;
    unsigned int* inst_flags;
    // colour-partitioned launches (null: all elements in one launch).  A pass then runs one
    // launch per element colour; elements of one colour share no node, so every K entry and
    // f_int entry receives at most one red.global.add per launch and its sum runs in colour
    // order: the same inputs give the same bits on every run.
    const int* order;                  // element indices of this launch's colour
    int ecount;                        // elements of this launch
};

// PCG scalars kept on the device (no host round trip per iteration)
struct CgScalars {
    double rhs_norm2, threshold;
    double abs_new, pq, alpha, rr, rz, beta;
    double rr_cap;  // mixed reliable updates: recurrence r.r above which a cycle has diverged
    int iterations, max_iterations, done, status;
    unsigned int counter[4];  // last-block tickets of the reductions
};

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
};

}  // namespace nb2

struct nb2_ctx {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0;
    int N = 0, E = 0, npe = 0, nq = 0, nqp = 0, n = 0;
    long long nnzb = 0, nnz = 0;
    nb2_material mat{};

    // mesh + pattern
    double* X = nullptr;
    int* conn = nullptr;
    int* brp = nullptr;
    int* bcol = nullptr;
    int* slot = nullptr;
    std::vector<int> h_brp, h_bcol;  // host copy of the block pattern

    // values and vectors
    double* K64 = nullptr;
    float* K32 = nullptr;
    double* Kcsr = nullptr;  // CSR-ordered copy of K64 for host downloads
    double* u = nullptr;
    double* u_old = nullptr;
    double* fint = nullptr;
    double* fext = nullptr;
    double* rhs = nullptr;  // minus_residual
    double* du = nullptr;   // delta_d
    double* inc = nullptr;  // prescribed increment
    unsigned char* mask = nullptr;  // active Dirichlet DOFs
    double* Ge = nullptr;
    double* Ke = nullptr;

    // quadrature-point state
    double* ep = nullptr;
    double* epbar = nullptr;
    double* ep_old = nullptr;
    double* epbar_old = nullptr;
    double* sig = nullptr;
    double* dpar = nullptr;
    double* detF = nullptr;
    double* u_tan = nullptr;  // displacement of the last MODE_STORE pass (its geometry)

    // FP32 matrix-free tangent (mixed-precision PCG): per-element relative coordinates, per-point
    // coefficients, per-element products / diagonal contributions, node -> element-slot lists
    float* mf_d = nullptr;   // [E][npe*3]
    float* mf_c = nullptr;   // [kc][nqp]
    float* mf_ye = nullptr;  // [npe][E][3]: one plane per local node (coalesced on both sides)
    int* nadj_ptr = nullptr; // [N+1]
    int* nadj = nullptr;     // [E*npe] element slots e*npe + a, grouped by node
    int* nadj_pl = nullptr;  // [E*npe] the same slots as plane positions a*E + e of mf_ye
    // colour-partitioned launches (hex8, single problem): elements grouped by colour
    int* corder = nullptr;                   // [E] elements sorted by colour
    std::vector<int> h_coff;                 // colour offsets into corder
    int colour_state = 0;  // 0 not set up, 1 ready, -1 not applicable (tet4, > 64 colours)
    int scatter = NB2_SCATTER_RED;  // element-pass launch mode (nb2_set_scatter_mode)
    bool newton_scatter = false;    // set while nb2_static_solve runs: colour-partitioned
    cudaGraphExec_t graph_mf = nullptr;

    // PCG workspace (FP64 and FP32 views share nothing)
    double *cg_x = nullptr, *cg_r = nullptr, *cg_p = nullptr, *cg_q = nullptr, *cg_inv = nullptr;
    float *cg32_x = nullptr, *cg32_r = nullptr, *cg32_p = nullptr, *cg32_q = nullptr,
          *cg32_inv = nullptr;
    double* partials = nullptr;  // reduction partials
    nb2::CgScalars* cgs = nullptr;
    nb2::CgScalars* h_cgs = nullptr;  // pinned mirror
    double* norms = nullptr;          // device norm results
    double* h_norms = nullptr;        // pinned mirror
    nb2::DeviceStatus* status = nullptr;

    // captured CG iteration blocks; the FP64 one per K buffer (the graph holds the K pointer)
    cudaGraphExec_t graph64[2] = {nullptr, nullptr}, graph32 = nullptr;
    // double-buffered K zeroing (FP64 stiffness passes of one problem): while a pass assembles
    // into K64, the previous K (K64_alt) is zeroed on zstream for the next pass
    double* K64_alt = nullptr;
    int kbuf = 0;            // which of the two buffers K64 is (selects graph64)
    bool alt_zeroed = false; // K64_alt's zeroing is queued (zev_done marks its end)
    int kalt_state = 0;      // 0 not set up, 1 ready, -1 off (the second buffer did not fit)
    cudaStream_t zstream = nullptr;
    cudaEvent_t zev_free = nullptr, zev_done = nullptr;

    // batched solves: set for the duration of one (device arrays owned by the batch state)
    const int* e_inst = nullptr;
    const int* inst_on = nullptr;
    unsigned int* inst_flags = nullptr;
    int batch_rows = 0, batch_lanes = 0;  // autotuned chunk rows / lanes per block row (0: default)

    long long launches = 0;
    std::string error;
};

namespace nb2 {

// launch geometry of the reduction kernels: persistent grid, fixed partial count
constexpr int kRedThreads = 256;
int reduction_blocks(const nb2_ctx* c);

// CUDA error -> context message + status
int cuda_fail(nb2_ctx* c, cudaError_t e, const char* what);
#define NB2_CUDA(ctx, call)                                     \
    do {                                                        \
        cudaError_t _e = (call);                                \
        if (_e != cudaSuccess) return nb2::cuda_fail(ctx, _e, #call); \
    } while (0)

#define NB2_TRY(x)                   \
    do {                             \
        int _s = (x);                \
        if (_s != NB2_OK) return _s; \
    } while (0)

// api.cu: lazily allocated buffers and the element status word
int ensure_k64(nb2_ctx* c);            // K64
int ensure_k64_alt(nb2_ctx* c);        // the second K buffer, its stream and events
int ensure_k32(nb2_ctx* c);            // K32 and the FP32 CG vectors
int ensure_cg32(nb2_ctx* c);           // the FP32 CG vectors only (matrix-free mixed PCG)
int ensure_split_buffers(nb2_ctx* c);  // stored quadrature-point outputs + their displacement
int reset_status(nb2_ctx* c);
int read_status(nb2_ctx* c);           // synchronises; the status code + neon's message

// pattern.cu
int build_pattern(nb2_ctx* c);
int build_node_adjacency(nb2_ctx* c);  // nadj_ptr / nadj
int ensure_colouring(nb2_ctx* c);      // element colours and the colour-sorted element list
int export_csr_values(nb2_ctx* c, const double* Kbsr, double* Kcsr_dev);

// elements.cu
int launch_element_kernel(nb2_ctx* c, int mode, int precision);
int launch_apply(nb2_ctx* c, const double* v, double* y);  // y = K v, FP64 matrix-free
int launch_element_stiffness(nb2_ctx* c, long long e, double* Ke_dev);  // one dense K_e
int launch_adjoint_shear(nb2_ctx* c, const double* lam, double* dJdG);
int launch_force_jvp(nb2_ctx* c, const double* v, double* y);  // exact (d f_int/du) v
int launch_mf_setup(nb2_ctx* c);  // FP32 matrix-free data + diagonal contributions
int mf_coefficients(int model);   // FP32 coefficients per quadrature point
void enqueue_apply32(nb2_ctx* c, const float* v, float* ye, const int* done);
void element_flop_model(const nb2_ctx* c, double* flops_per_element);

// pcg.cu
struct BsrView {
    const int* brp;
    const int* bcol;
    int nrows_block;  // N
};
int pcg_device_fp64(nb2_ctx* c, const double* b, double* x, double tol, int maxit, bool use_mask,
                    int* iterations, double* error, bool use_graphs);
int pcg_device_fp32(nb2_ctx* c, const double* b, double* x, double tol, int maxit, int* iterations,
                    double* error, bool use_graphs);
// mixed precision with reliable updates: FP32 iterations on K32, FP64 true residual (matrix-free
// stored tangent) every `delta` reduction; work: n doubles
int pcg_reliable_mixed(nb2_ctx* c, const double* b, double* x, double tol, double delta,
                       int maxit, double* work, int* iterations, bool use_graphs,
                       bool matrix_free);
int ensure_mf(nb2_ctx* c);  // FP32 matrix-free buffers + node adjacency
int mf_apply(nb2_ctx* c, const double* v, double* y);  // FP32 matrix-free K v (device FP64)
int pcg_csr_host(int n, const int* rowptr, const int* col, const double* val, const double* b,
                 double* x, double tol, int maxit, int* iterations, double* error,
                 std::string* err);
void release_graphs(nb2_ctx* c);
void bsr_spmv_fp64(nb2_ctx* c, const double* x, double* y, bool use_mask);
void bsr_spmv_mixed_accum(nb2_ctx* c, const double* x, double* y);  // y = K32 x in FP64 accum
// five norms ||du||, ||u||, ||rhs||, ||fext||, ||fint|| into c->h_norms (synchronises)
int compute_norms(nb2_ctx* c);
double device_dot_sync(nb2_ctx* c, const double* a, const double* b, int n);

}  // namespace nb2
