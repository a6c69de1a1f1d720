// neon_oracle.cpp -- CPU oracle (test infrastructure, NOT the product).
//
// A C++17 + OpenMP, FP64 restatement of dbeurle/neon's solid-mechanics Newton step, used
// (1) as the parity checker for the CUDA path and (2) as the timed CPU baseline.  It is never
// linked into the product library; only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg / reference arm load it.
//
// The reference cannot be built in this environment (Eigen, TBB, nlohmann-json, range-v3,
// Boost, VTK ... are absent), so this file restates its algorithm.  Every function cites the
// reference file:line it follows.  Parity pins: the reference's own known-answer tests
// (test/*.cpp), restated in tests/golden/kats.json and checked by tests/test_oracle_kats.py.
//
// Parallel structure mirrors the reference so the CPU timing is representative:
//   * element loop of the stiffness assembly is parallel, each entry is added with a binary
//     search into the CSR row plus an atomic add (static_matrix.hpp:243-277,
//     thread_safe_plugin.hpp:7-23);
//   * internal-force gather is serial (static_matrix.hpp:189-203);
//   * deformation-measure update is parallel over elements (submesh.cpp:210-237), the
//     determinant check is serial (submesh.cpp:239-269);
//   * J2 and microsphere updates are parallel over quadrature points, the linear-elastic and
//     neo-Hookean updates are serial transforms (model files);
//   * the CG SpMV is parallel (Eigen's OpenMP row-major sparse*dense product), vector ops are
//     serial, RCM is computed once and P^T A P is rebuilt on every solve
//     (linear_solver.cpp:39-109).
//
// Third-party arithmetic restated here (Eigen, pinned at hg a67d661 by
// external/eigen3/CMakeLists.txt:10): SparseMatrix::setFromTriplets (sorted unique columns per
// row, explicit zeros kept), ConjugateGradient + DiagonalPreconditioner (the published PCG
// algorithm with ||r||^2 < max(tol^2 ||b||^2, DBL_MIN) as the stopping test and invdiag = 1 for
// a zero diagonal), fixed-size 3x3 determinant (first-row cofactor expansion) and inverse
// (cofactors scaled by 1/det, det from the first column).  Boost.Math relative_difference
// (used by neon's is_approx, numeric/float_compare.hpp:20-32) is restated in is_approx_zero().

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline double wtime() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ----------------------------------------------------------------------------------------
// Status codes (same numbering as the product's C-ABI, include/neon_b200.h)
// ----------------------------------------------------------------------------------------
enum : int {
    ORC_OK = 0,
    ORC_E_NEG_DETJ = 1,
    ORC_E_NAN = 2,
    ORC_E_RETURN_MAP = 3,
    ORC_E_CG_MAXIT = 4,
    ORC_E_INPUT = 7,
    ORC_E_NEWTON_MAXIT = 9,
    ORC_E_CUTBACK_LIMIT = 10,
};

enum : int {
    LINEAR_ELASTIC = 0,
    NEO_HOOKE = 1,
    J2_SMALL_STRAIN = 2,
    GAUSS_AFFINE_MICROSPHERE = 3,
    LANGEVIN_AFFINE_MICROSPHERE = 4,
    NONAFFINE_MICROSPHERE = 5
};

// ----------------------------------------------------------------------------------------
// 3x3 helpers, row-major double[9]
// ----------------------------------------------------------------------------------------
// Fixed-size determinant by first-row cofactor expansion, evaluated as
// h(0,1,2) - h(1,0,2) + h(2,0,1) with h(a,b,c) = m(0,a) (m(1,b) m(2,c) - m(1,c) m(2,b)).
inline double det3(const double* m) {
    auto h = [&](int a, int b, int c) {
        return m[0 * 3 + a] * (m[1 * 3 + b] * m[2 * 3 + c] - m[1 * 3 + c] * m[2 * 3 + b]);
    };
    return h(0, 1, 2) - h(1, 0, 2) + h(2, 0, 1);
}

// Inverse by cofactors: inv(i,j) = cof(j,i) / det, det = sum_i cof(i,0) m(i,0).
inline void inv3(const double* m, double* r) {
    auto M = [&](int i, int j) { return m[i * 3 + j]; };
    auto cof = [&](int i, int j) {
        int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        return M(i1, j1) * M(i2, j2) - M(i1, j2) * M(i2, j1);
    };
    double c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
    double det = c00 * M(0, 0) + c10 * M(1, 0) + c20 * M(2, 0);
    double invdet = 1.0 / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i * 3 + j] = cof(j, i) * invdet;
}

inline void matmul3(const double* a, const double* b, double* c) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += a[i * 3 + k] * b[k * 3 + j];
            c[i * 3 + j] = s;
        }
}

inline double trace3(const double* a) { return a[0] + a[4] + a[8]; }

inline void deviatoric3(const double* a, double* d) {
    // tensor_operations.hpp:33-43: a - I tr(a)/3
    double v = trace3(a) / 3.0;
    for (int i = 0; i < 9; ++i) d[i] = a[i];
    d[0] -= v;
    d[4] -= v;
    d[8] -= v;
}

inline double norm3(const double* a) {
    double s = 0.0;
    for (int i = 0; i < 9; ++i) s += a[i] * a[i];
    return std::sqrt(s);
}

// stress_routines.hpp:25-28: sqrt(3/2) |dev(a)|
inline double von_mises(const double* s) {
    double d[9];
    deviatoric3(s, d);
    return std::sqrt(3.0 / 2.0) * norm3(d);
}

// stress_routines.hpp:37-42: lambda tr(e) I + 2 G e
inline void cauchy_stress_linear(double G, double lambda, const double* e, double* s) {
    double tr = trace3(e);
    for (int i = 0; i < 9; ++i) s[i] = 2.0 * G * e[i];
    s[0] += lambda * tr;
    s[4] += lambda * tr;
    s[8] += lambda * tr;
}

// kinetic Voigt (tensor_operations.hpp:337-340): (a00, a11, a22, a12, a02, a01)
inline void kinetic_voigt(const double* a, double* v) {
    v[0] = a[0];
    v[1] = a[4];
    v[2] = a[8];
    v[3] = a[5];
    v[4] = a[2];
    v[5] = a[1];
}

// 6x6 isotropic Voigt tangent with engineering shears (isotropic_linear_elasticity.cpp:55-67)
inline void isotropic_voigt(double lambda, double mu, double* D) {
    for (int i = 0; i < 36; ++i) D[i] = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D[i * 6 + j] = lambda;
    for (int i = 0; i < 3; ++i) D[i * 6 + i] = lambda + 2.0 * mu;
    for (int i = 3; i < 6; ++i) D[i * 6 + i] = mu;
}

// Boost.Math relative_difference(x, 0) <= 1e-10 || |x| <= abs_tol  (float_compare.hpp:20-32)
inline bool is_approx_zero(double x, double abs_tol) {
    double rd;
    double maxv = std::numeric_limits<double>::max();
    double minv = std::numeric_limits<double>::min();
    if (std::isnan(x)) {
        rd = maxv;
    } else if (std::fabs(x) > maxv) {
        rd = maxv;
    } else {
        double a = std::fabs(x), b = 0.0;
        if (a < minv) a = minv;
        if (b < minv) b = minv;
        rd = std::max(std::fabs((a - b) / a), std::fabs((a - b) / b));
    }
    return rd <= 1e-10 || std::fabs(x) <= abs_tol;
}

// ----------------------------------------------------------------------------------------
// Shape functions and quadrature
// ----------------------------------------------------------------------------------------
struct Interpolation {
    int npe = 0, nq = 0;
    std::vector<double> dN;  // [nq][npe][3]
    std::vector<double> w;   // [nq]
};

// interpolations/hexahedron.cpp:10-67 with quadrature/hexahedron/hexahedron_quadrature.cpp:27-40
Interpolation make_hex8() {
    Interpolation I;
    I.npe = 8;
    I.nq = 8;
    const double lc[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                             {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    const double qp = 1.0 / std::sqrt(3.0);
    const double qc[8][3] = {{-qp, -qp, -qp}, {qp, -qp, -qp}, {qp, qp, -qp}, {-qp, qp, -qp},
                             {-qp, -qp, qp},  {qp, -qp, qp},  {qp, qp, qp},  {-qp, qp, qp}};
    I.dN.resize(8 * 8 * 3);
    I.w.assign(8, 1.0);
    for (int l = 0; l < 8; ++l) {
        double xi = qc[l][0], eta = qc[l][1], zeta = qc[l][2];
        for (int a = 0; a < 8; ++a) {
            double xa = lc[a][0], ea = lc[a][1], za = lc[a][2];
            double* d = &I.dN[(l * 8 + a) * 3];
            d[0] = 1.0 / 8.0 * xa * (1.0 + ea * eta) * (1.0 + za * zeta);
            d[1] = 1.0 / 8.0 * (1.0 + xa * xi) * ea * (1.0 + za * zeta);
            d[2] = 1.0 / 8.0 * (1.0 + xa * xi) * (1.0 + ea * eta) * za;
        }
    }
    return I;
}

// interpolations/tetrahedron.cpp:6-45 with the 1-point rule of
// quadrature/tetrahedron/tetrahedron_quadrature.cpp:12-17 (weights / 6, :74-77)
Interpolation make_tet4() {
    Interpolation I;
    I.npe = 4;
    I.nq = 1;
    I.dN = {1, 0, 0, 0, 1, 0, 0, 0, 1, -1, -1, -1};
    I.w = {1.0 / 6.0};
    return I;
}

// Unit-sphere rules of the microsphere models (quadrature/sphere/unit_sphere_quadrature.cpp):
// BO21 (:10-31) and BO33 (:33-91), both from Bazant and Oh (1986), Table 1
struct SphereRule {
    int n = 0;
    double r[33][3];
    double w[33];
};

SphereRule make_bo21() {
    SphereRule s;
    const double w1 = 0.0265214244093 * 2.0, w2 = 0.0199301476312 * 2.0, w3 = 0.0250712367487 * 2.0;
    const double dc0 = 0.707106781187, dc1 = 0.387907304067, dc2 = 0.836095596749;
    const double pts[21][3] = {{1.0, 0.0, 0.0},   {0.0, 1.0, 0.0},    {0.0, 0.0, 1.0},
                               {dc0, dc0, 0.0},   {dc0, -dc0, 0.0},   {dc0, 0.0, dc0},
                               {dc0, 0.0, -dc0},  {0.0, dc0, dc0},    {0.0, dc0, -dc0},
                               {dc1, dc1, dc2},   {dc1, dc1, -dc2},   {dc1, -dc1, dc2},
                               {dc1, -dc1, -dc2}, {dc1, dc2, dc1},    {dc1, dc2, -dc1},
                               {dc1, -dc2, dc1},  {dc1, -dc2, -dc1},  {dc2, dc1, dc1},
                               {dc2, dc1, -dc1},  {dc2, -dc1, dc1},   {dc2, -dc1, -dc1}};
    s.n = 21;
    for (int i = 0; i < 21; ++i) {
        for (int k = 0; k < 3; ++k) s.r[i][k] = pts[i][k];
        s.w[i] = (i < 3) ? w1 : (i < 9 ? w2 : w3);
    }
    return s;
}

SphereRule make_bo33() {
    SphereRule s;
    const double w1 = 2.0 * 0.00985353993433, w2 = 2.0 * 0.0162969685886,
                 w3 = 2.0 * 0.0134788844008, w4 = 2.0 * 0.0175759129880;
    const double a = 0.707106781187, b = 0.933898956394, c = 0.357537045978, d = 0.437263676092,
                 e = 0.785875915868;
    const double pts[33][3] = {
        {1, 0, 0},  {0, 1, 0},   {0, 0, 1},                                         // 3 axes
        {a, a, 0},  {a, -a, 0},  {a, 0, a},  {a, 0, -a},  {0, a, a},  {0, a, -a},   // 6 edges
        {b, c, 0},  {b, -c, 0},  {c, b, 0},  {c, -b, 0},                            // 12 (b, c)
        {b, 0, c},  {b, 0, -c},  {c, 0, b},  {c, 0, -b},
        {0, b, c},  {0, b, -c},  {0, c, b},  {0, c, -b},
        {d, d, e},  {d, d, -e},  {d, -d, e}, {d, -d, -e},                           // 12 (d, e)
        {d, e, d},  {d, e, -d},  {d, -e, d}, {d, -e, -d},
        {e, d, d},  {e, d, -d},  {e, -d, d}, {e, -d, -d}};
    s.n = 33;
    for (int i = 0; i < 33; ++i) {
        for (int k = 0; k < 3; ++k) s.r[i][k] = pts[i][k];
        s.w[i] = i < 3 ? w1 : (i < 9 ? w2 : (i < 21 ? w3 : w4));
    }
    return s;
}

// ----------------------------------------------------------------------------------------
// Material
// ----------------------------------------------------------------------------------------
struct Material {
    int model = 0;
    double K = 0, G = 0;             // isotropic_elastic_property.cpp:10-43
    double sigma_y = 0, H_iso = 0;   // isotropic_elastic_plastic.cpp:10-38
    double segments = 0;             // micromechanical_elastomer.cpp:13-21
    double nonaffine_p = 0;          // nonaffine_microsphere.cpp:17-25
    int sphere_points = 21;          // unit-sphere rule of the microsphere models (BO21 / BO33)
    double lambda() const { return K - 2.0 * G / 3.0; }  // isotropic_elastic_property.hpp:28
};

// ----------------------------------------------------------------------------------------
// The mesh + internal-variable store (solid::mesh / solid::submesh / internal_variables)
// ----------------------------------------------------------------------------------------
struct Oracle {
    int N = 0, E = 0, npe = 0, nq = 0;
    std::vector<double> X;  // [N][3]
    std::vector<double> x;  // [N][3] current configuration
    std::vector<int> conn;  // [E][npe]
    Interpolation sf;
    Material mat;
    std::vector<double> Ge;  // optional per-element shear modulus (microsphere)
    SphereRule sphere = make_bo21();

    // CSR pattern (row-major, int32, sorted unique columns)
    std::vector<int> rowptr, col;

    // quadrature-point variables (internal_variables.hpp:22-234); index e*nq + l
    std::vector<double> H, F, detF, sigma, D, vm;  // H,F,sigma: 9/qp; D: 36/qp
    std::vector<double> ep, ep_old, epbar, epbar_old;  // J2 history (versioned)
    std::vector<double> sigma_old, F_old;               // versioned second-order tensors

    int ndofs() const { return 3 * N; }
    long long nnz() const { return (long long)col.size(); }
    double shear(int e) const { return Ge.empty() ? mat.G : Ge[e]; }
};

// sparsity_pattern.hpp:18-48: setFromTriplets of every (dof_p, dof_q) pair of every element
// yields, per row, the sorted unique set of coupled columns.  Built here from node adjacency
// (identical result: all 3x3 DOF pairs of every node pair sharing an element are present).
void build_pattern(Oracle& o) {
    std::vector<std::vector<int>> adj(o.N);
    for (int e = 0; e < o.E; ++e) {
        const int* c = &o.conn[(size_t)e * o.npe];
        for (int a = 0; a < o.npe; ++a)
            for (int b = 0; b < o.npe; ++b) adj[c[a]].push_back(c[b]);
    }
    for (auto& v : adj) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    }
    int n = 3 * o.N;
    o.rowptr.assign(n + 1, 0);
    for (int a = 0; a < o.N; ++a)
        for (int r = 0; r < 3; ++r) o.rowptr[3 * a + r + 1] = 3 * (int)adj[a].size();
    for (int i = 0; i < n; ++i) o.rowptr[i + 1] += o.rowptr[i];
    o.col.resize(o.rowptr[n]);
    for (int a = 0; a < o.N; ++a)
        for (int r = 0; r < 3; ++r) {
            int p = o.rowptr[3 * a + r];
            for (int b : adj[a])
                for (int c = 0; c < 3; ++c) o.col[p++] = 3 * b + c;
        }
}

// ----------------------------------------------------------------------------------------
// Constitutive updates (per quadrature point)
// ----------------------------------------------------------------------------------------

// isotropic_linear_elasticity.cpp:27-53
void update_linear_elastic(Oracle& o, size_t q) {
    const double* Hq = &o.H[q * 9];
    double eps[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) eps[i * 3 + j] = 0.5 * (Hq[i * 3 + j] + Hq[j * 3 + i]);
    cauchy_stress_linear(o.mat.G, o.mat.lambda(), eps, &o.sigma[q * 9]);
    o.vm[q] = von_mises(&o.sigma[q * 9]);
    isotropic_voigt(o.mat.lambda(), o.mat.G, &o.D[q * 36]);
}

// compressible_neohooke.cpp:17-90
void update_neo_hooke(Oracle& o, size_t q) {
    const double* Fq = &o.F[q * 9];
    double J = o.detF[q];
    double lambda = o.mat.lambda(), mu = o.mat.G;
    double B[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += Fq[i * 3 + k] * Fq[j * 3 + k];
            B[i * 3 + j] = s;
        }
    double* s = &o.sigma[q * 9];
    double lnJ = std::log(J);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double I = (i == j) ? 1.0 : 0.0;
            s[i * 3 + j] = (lambda * lnJ * I + mu * (B[i * 3 + j] - I)) / J;
        }
    isotropic_voigt(lambda, mu - lambda * std::log(J), &o.D[q * 36]);
}

// small_strain_J2_plasticity.cpp:30-163 (radial return, algorithmic tangent).  The plastic
// strain and accumulated plastic strain of the *current* state are mutated on every call.
int update_j2(Oracle& o, size_t q) {
    const double G = o.mat.G, lambda = o.mat.lambda();
    const double Hh = o.mat.H_iso;
    auto yield = [&](double ebar) { return o.mat.sigma_y + ebar * Hh; };
    auto f_yield = [&](double vm, double ebar, double dg) {
        return (vm - 3.0 * G * dg) - yield(ebar + dg);
    };
    const double* Hq = &o.H[q * 9];
    double eps[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) eps[i * 3 + j] = 0.5 * (Hq[i * 3 + j] + Hq[j * 3 + i]);
    double* epq = &o.ep[q * 9];
    double& ebar = o.epbar[q];
    double* s = &o.sigma[q * 9];
    double ee[9];
    for (int i = 0; i < 9; ++i) ee[i] = eps[i] - epq[i];
    cauchy_stress_linear(G, lambda, ee, s);
    double vm = von_mises(s);
    o.vm[q] = vm;
    double* Dq = &o.D[q * 36];
    if (f_yield(vm, ebar, 0.0) <= 0.0) {
        isotropic_voigt(lambda, G, Dq);
        return ORC_OK;
    }
    const double vm_trial = vm;
    double dev[9];
    deviatoric3(s, dev);
    double dn = norm3(dev);
    double nrm[9];
    for (int i = 0; i < 9; ++i) nrm[i] = dev[i] / dn;
    // perform_radial_return (:108-155)
    double dg = 0.0;
    double f = f_yield(vm, ebar, 0.0);
    int it = 0;
    while (f > 1.0e-6 && it < 50) {
        double Hm = Hh;
        double ddg = f / (3.0 * G + Hm);
        dg += ddg;
        f = f_yield(vm, ebar, dg);
        ++it;
    }
    if (it == 50) return ORC_E_RETURN_MAP;
    const double s32 = std::sqrt(3.0 / 2.0);
    for (int i = 0; i < 9; ++i) epq[i] += dg * s32 * nrm[i];
    for (int i = 0; i < 9; ++i) s[i] -= 2.0 * G * dg * s32 * nrm[i];
    o.vm[q] = von_mises(s);
    ebar += dg;
    // algorithmic_tangent (:95-106)
    double Ce[36];
    isotropic_voigt(lambda, G, Ce);
    const double Idev[36] = {2.0 / 3.0,  -1.0 / 3.0, -1.0 / 3.0, 0, 0, 0,  //
                             -1.0 / 3.0, 2.0 / 3.0,  -1.0 / 3.0, 0, 0, 0,  //
                             -1.0 / 3.0, -1.0 / 3.0, 2.0 / 3.0,  0, 0, 0,  //
                             0, 0, 0, 0.5, 0, 0, 0, 0, 0, 0, 0.5, 0, 0, 0, 0, 0, 0, 0.5};
    double nv[6];
    kinetic_voigt(nrm, nv);
    double c1 = dg * 6.0 * std::pow(G, 2) / vm_trial;
    double c2 = 6.0 * std::pow(G, 2) * (dg / vm_trial - 1.0 / (3.0 * G + Hh));
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j)
            Dq[i * 6 + j] = Ce[i * 6 + j] - c1 * Idev[i * 6 + j] + c2 * (nv[i] * nv[j]);
    return ORC_OK;
}

// gaussian_affine_microsphere.cpp:23-88, volumetric_free_energy.hpp:16-30,
// detail/microsphere.hpp:16-20, tensor_operations.hpp:70-73 (unimodular).
// langevin: affine_microsphere.cpp:23-112 -- the chain force and stiffness follow the Pade
// approximants of the inverse Langevin function (detail/microsphere.hpp:40-70):
//   macro stress  G sum_i w_i pade_first(l_i, N) t_i (x) t_i,
//   macro moduli  G sum_i w_i l_i^-2 (pade_second - pade_first) t_i (x) t_i (x) t_i (x) t_i,
// with l_i = |t_i|; the Gaussian model has 3 G sum_i w_i t_i (x) t_i and zero macro moduli.
double pade_first(double l, double N) { return (3.0 * N - std::pow(l, 2)) / (N - std::pow(l, 2)); }
double pade_second(double l, double N) {
    return (std::pow(l, 4) + 3.0 * std::pow(N, 2)) / std::pow(N - std::pow(l, 2), 2);
}

void microsphere_response(Oracle& o, size_t q, const double* tau, const double* macroC);

void update_microsphere(Oracle& o, size_t q, double G, bool langevin = false) {
    const double Nseg = o.mat.segments;
    const double* Fq = &o.F[q * 9];
    double scale = std::pow(det3(Fq), -1.0 / 3.0);
    double Fb[9];
    for (int i = 0; i < 9; ++i) Fb[i] = scale * Fq[i];
    // compute_macro_stress: 3 G sum_i w_i t_i (x) t_i, t_i = Fbar r_i (Gaussian), or
    // G sum_i w_i pade_first t_i (x) t_i (Langevin); compute_macro_moduli (Langevin)
    double acc[9] = {0};
    double macroC[36] = {0};
    for (int i = 0; i < o.sphere.n; ++i) {
        double t[3];
        for (int a = 0; a < 3; ++a)
            t[a] = Fb[a * 3 + 0] * o.sphere.r[i][0] + Fb[a * 3 + 1] * o.sphere.r[i][1] +
                   Fb[a * 3 + 2] * o.sphere.r[i][2];
        double f = 1.0;
        if (langevin) {
            const double l = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
            f = pade_first(l, Nseg);
            const double a4 = std::pow(l, -2) * (pade_second(l, Nseg) - pade_first(l, Nseg));
            double tt[9], tv[6];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) tt[a * 3 + b] = t[a] * t[b];
            kinetic_voigt(tt, tv);
            for (int a = 0; a < 6; ++a)
                for (int b = 0; b < 6; ++b) macroC[a * 6 + b] += (a4 * tv[a] * tv[b]) * o.sphere.w[i];
        }
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) acc[a * 3 + b] += (f * t[a] * t[b]) * o.sphere.w[i];
    }
    double tau[9];
    for (int i = 0; i < 9; ++i) tau[i] = (langevin ? G : 3.0 * G) * acc[i];
    for (int i = 0; i < 36; ++i) macroC[i] *= G;
    microsphere_response(o, q, tau, macroC);
}

// affine_microsphere::compute_kirchhoff_stress and compute_material_tangent
// (affine_microsphere.cpp:55-77), shared by the affine and non-affine models
void microsphere_response(Oracle& o, size_t q, const double* tau, const double* macroC) {
    const double K = o.mat.K;
    const double J = o.detF[q];
    const double pressure = J * (K / 2.0 * (J - 1.0 / J));
    // Kirchhoff stress p I + dev(tau) -> Cauchy / J
    double dev[9];
    deviatoric3(tau, dev);
    double* s = &o.sigma[q * 9];
    for (int i = 0; i < 9; ++i) s[i] = dev[i];
    s[0] += pressure;
    s[4] += pressure;
    s[8] += pressure;
    for (int i = 0; i < 9; ++i) s[i] /= J;
    // compute_material_tangent (macro moduli zero for the Gaussian model)
    double kappa = std::pow(J, 2) * (K / 2.0 * (1.0 + 1.0 / std::pow(J, 2)));
    double tv[6];
    kinetic_voigt(tau, tv);
    const double one[6] = {1, 1, 1, 0, 0, 0};
    const double Ikin[6] = {1, 1, 1, 0.5, 0.5, 0.5};  // kinematic identity / fourth_order_identity
    double trt = trace3(tau);
    double Dbar[36];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double Iij = (i == j) ? Ikin[i] : 0.0;
            Dbar[i * 6 + j] = macroC[i * 6 + j] + 2.0 / 3.0 * trt * Iij -
                              2.0 / 3.0 * (tv[i] * one[j] + one[i] * tv[j]);
        }
    // P = kinetic deviatoric (shear diagonal 1)
    double P[36] = {0};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) P[i * 6 + j] = (i == j) ? 2.0 / 3.0 : -1.0 / 3.0;
    for (int i = 3; i < 6; ++i) P[i * 6 + i] = 1.0;
    double PD[36], PDP[36];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double v = 0;
            for (int k = 0; k < 6; ++k) v += P[i * 6 + k] * Dbar[k * 6 + j];
            PD[i * 6 + j] = v;
        }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double v = 0;
            for (int k = 0; k < 6; ++k) v += PD[i * 6 + k] * P[k * 6 + j];
            PDP[i * 6 + j] = v;
        }
    double* Dq = &o.D[q * 36];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double IoI = (i < 3 && j < 3) ? 1.0 : 0.0;
            double I = (i == j) ? Ikin[i] : 0.0;
            Dq[i * 6 + j] = (kappa + pressure) * IoI - 2.0 * pressure * I + PDP[i * 6 + j];
        }
}

// nonaffine_microsphere.cpp:29-175 (members nonaffine_microsphere.hpp: effective tube geometry
// U = 9, tube parameter q = 1; the stretch parameter p from the material).  Chain part on the
// non-affine stretch lambda = (sum_i w_i |t_i|^p)^(1/p), tube part on the deformed normals
// n_i = Fbar^-T r_i (area stretch nu_i = |n_i|):
//   h = sum w |t|^(p-2) t(x)t,  H = (p-2) sum w |t|^(p-4) t(x)t(x)t(x)t,
//   k = q sum w nu^(q-2) n(x)n,  K = q(q-2) sum w nu^(q-4) n(x)n(x)n(x)n,
//   G = 2q sum w nu^(q-2) o(n)   (o: compute_o_dot_product),
//   tau = G pf lambda^(2-p) h - G N U k,
//   C = (G ps lambda^(2-2p) - (p-1) G pf lambda^(2-2p)) h(x)h + G pf lambda^(2-p) H
//       + G N U (K + G),
// with pf, ps the Pade approximants at lambda; then the affine model's stress and tangent.
void o_dot_product(const double* n, double* o6) {
    const double n0 = n[0], n1 = n[1], n2 = n[2];
    const double m[36] = {2.0 * n0 * n0, 0.0, 0.0, 0.0, n0 * n2, n0 * n1,
                          0.0, 2.0 * n1 * n1, 0.0, n1 * n2, 0.0, n0 * n1,
                          0.0, 0.0, 2.0 * n2 * n2, n1 * n2, n0 * n2, 0.0,
                          0.0, n1 * n2, n1 * n2, 0.5 * (n1 * n1 + n2 * n2), 0.5 * n0 * n1, 0.5 * n0 * n2,
                          n0 * n2, 0.0, n0 * n2, 0.5 * n0 * n1, 0.5 * (n0 * n0 + n2 * n2), 0.5 * n2 * n1,
                          n0 * n1, n0 * n1, 0.0, 0.5 * n0 * n2, 0.5 * n2 * n1, 0.5 * (n0 * n0 + n1 * n1)};
    for (int i = 0; i < 36; ++i) o6[i] = m[i];
}

void update_nonaffine(Oracle& o, size_t q, double G) {
    const double N = o.mat.segments, p = o.mat.nonaffine_p;
    const double U = 9.0, qt = 1.0;  // effective_tube_geometry, non_affine_tube_parameter
    const double* Fq = &o.F[q * 9];
    const double scale = std::pow(det3(Fq), -1.0 / 3.0);
    double Fb[9], Fbi[9];
    for (int i = 0; i < 9; ++i) Fb[i] = scale * Fq[i];
    inv3(Fb, Fbi);
    double lp = 0.0, h[9] = {0}, H[36] = {0}, k[9] = {0}, KG[36] = {0};
    for (int i = 0; i < o.sphere.n; ++i) {
        const double* r = o.sphere.r[i];
        const double w = o.sphere.w[i];
        double t[3], n[3];
        for (int a = 0; a < 3; ++a) {
            t[a] = Fb[a * 3 + 0] * r[0] + Fb[a * 3 + 1] * r[1] + Fb[a * 3 + 2] * r[2];
            n[a] = Fbi[0 * 3 + a] * r[0] + Fbi[1 * 3 + a] * r[1] + Fbi[2 * 3 + a] * r[2];
        }
        const double l = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        const double nu = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        lp += std::pow(l, p) * w;
        double tt[9], nn[9], tv[6], nv[6], od[36];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                tt[a * 3 + b] = t[a] * t[b];
                nn[a * 3 + b] = n[a] * n[b];
            }
        kinetic_voigt(tt, tv);
        kinetic_voigt(nn, nv);
        o_dot_product(n, od);
        for (int a = 0; a < 9; ++a) {
            h[a] += std::pow(l, p - 2.0) * tt[a] * w;
            k[a] += std::pow(nu, qt - 2.0) * nn[a] * w;
        }
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b) {
                H[a * 6 + b] += std::pow(l, p - 4.0) * (tv[a] * tv[b]) * w;
                KG[a * 6 + b] += qt * (qt - 2.0) * std::pow(nu, qt - 4.0) * (nv[a] * nv[b]) * w +
                                 2.0 * qt * std::pow(nu, qt - 2.0) * od[a * 6 + b] * w;
            }
    }
    const double lam = std::pow(lp, 1.0 / p);
    for (int a = 0; a < 36; ++a) H[a] *= (p - 2.0);
    for (int a = 0; a < 9; ++a) k[a] *= qt;
    const double micro_tau = G * pade_first(lam, N) * lam;
    const double micro_C = G * pade_second(lam, N);
    double tau[9], hv[6], C[36];
    kinetic_voigt(h, hv);
    for (int a = 0; a < 9; ++a)
        tau[a] = micro_tau * std::pow(lam, 1.0 - p) * h[a] - G * N * U * k[a];
    const double chh = micro_C * std::pow(lam, 2.0 - 2.0 * p) -
                       (p - 1.0) * micro_tau * std::pow(lam, 1.0 - 2.0 * p);
    for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b)
            C[a * 6 + b] = chh * (hv[a] * hv[b]) + micro_tau * std::pow(lam, 1.0 - p) * H[a * 6 + b] +
                           G * N * U * KG[a * 6 + b];
    microsphere_response(o, q, tau, C);
}

// ----------------------------------------------------------------------------------------
// solid::mesh::update_internal_variables (mesh.cpp:56-70) -> submesh (submesh.cpp:194-269)
// ----------------------------------------------------------------------------------------
int update_internal_variables(Oracle& o, const double* u, std::string* msg) {
    // material_coordinates.cpp:23-27: x = u; x += X
    for (int i = 0; i < 3 * o.N; ++i) o.x[i] = u[i] + o.X[i];
    // update_deformation_measures (submesh.cpp:210-237), parallel over elements
    const int npe = o.npe, nq = o.nq;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < o.E; ++e) {
        const int* c = &o.conn[(size_t)e * npe];
        for (int l = 0; l < nq; ++l) {
            const double* dN = &o.sf.dN[(size_t)l * npe * 3];
            double F0[9] = {0}, Fc[9] = {0}, U[9] = {0};
            for (int a = 0; a < npe; ++a) {
                const double* Xa = &o.X[(size_t)c[a] * 3];
                const double* xa = &o.x[(size_t)c[a] * 3];
                for (int i = 0; i < 3; ++i)
                    for (int k = 0; k < 3; ++k) {
                        F0[i * 3 + k] += Xa[i] * dN[a * 3 + k];
                        Fc[i * 3 + k] += xa[i] * dN[a * 3 + k];
                    }
            }
            double F0i[9];
            inv3(F0, F0i);
            // B_0t = dN F0^-1 (npe x 3); H = (x - X) B_0t
            for (int a = 0; a < npe; ++a) {
                double b0[3];
                for (int k = 0; k < 3; ++k)
                    b0[k] = dN[a * 3 + 0] * F0i[0 * 3 + k] + dN[a * 3 + 1] * F0i[1 * 3 + k] +
                            dN[a * 3 + 2] * F0i[2 * 3 + k];
                const double* Xa = &o.X[(size_t)c[a] * 3];
                const double* xa = &o.x[(size_t)c[a] * 3];
                for (int i = 0; i < 3; ++i)
                    for (int k = 0; k < 3; ++k) U[i * 3 + k] += (xa[i] - Xa[i]) * b0[k];
            }
            size_t q = (size_t)e * nq + l;
            for (int i = 0; i < 9; ++i) o.H[q * 9 + i] = U[i];
            matmul3(Fc, F0i, &o.F[q * 9]);
        }
    }
    // update_Jacobian_determinants (submesh.cpp:239-269), serial
    size_t nqp = (size_t)o.E * nq;
    long long first = -1, count = 0;
    for (size_t q = 0; q < nqp; ++q) {
        o.detF[q] = det3(&o.F[q * 9]);
        if (std::signbit(o.detF[q])) {
            if (first < 0) first = (long long)q;
            ++count;
        }
    }
    if (first >= 0) {
        if (msg) {
            char buf[256];
            std::snprintf(buf, sizeof buf,
                          "Positive Jacobian assumption violated at element %lld and local "
                          "quadrature point %lld (%g), another %lld violations found",
                          first / nq, first % nq, o.detF[first], count - 1);
            *msg = buf;
        }
        return ORC_E_NEG_DETJ;
    }
    // constitutive update
    int status = ORC_OK;
    switch (o.mat.model) {
        case LINEAR_ELASTIC:
            for (size_t q = 0; q < nqp; ++q) update_linear_elastic(o, q);
            break;
        case NEO_HOOKE:
            for (size_t q = 0; q < nqp; ++q) update_neo_hooke(o, q);
            break;
        case J2_SMALL_STRAIN: {
            std::atomic<int> bad{0};
#pragma omp parallel for schedule(static)
            for (long long q = 0; q < (long long)nqp; ++q)
                if (update_j2(o, (size_t)q) != ORC_OK) bad = 1;
            if (bad) {
                status = ORC_E_RETURN_MAP;
                if (msg) *msg = "Non-convergence in radial return method.";
            }
            break;
        }
        case GAUSS_AFFINE_MICROSPHERE:
#pragma omp parallel for schedule(static)
            for (long long q = 0; q < (long long)nqp; ++q)
                update_microsphere(o, (size_t)q, o.shear((int)(q / o.nq)));
            break;
        case LANGEVIN_AFFINE_MICROSPHERE:
#pragma omp parallel for schedule(static)
            for (long long q = 0; q < (long long)nqp; ++q)
                update_microsphere(o, (size_t)q, o.shear((int)(q / o.nq)), true);
            break;
        case NONAFFINE_MICROSPHERE:
#pragma omp parallel for schedule(static)
            for (long long q = 0; q < (long long)nqp; ++q)
                update_nonaffine(o, (size_t)q, o.shear((int)(q / o.nq)));
            break;
    }
    if (status != ORC_OK) return status;
    // FE_INVALID check (submesh.cpp:196-207) restated as a NaN scan of the outputs
    for (size_t q = 0; q < nqp; ++q)
        for (int i = 0; i < 9; ++i)
            if (std::isnan(o.sigma[q * 9 + i])) {
                if (msg) *msg = "Floating point error reported";
                return ORC_E_NAN;
            }
    return ORC_OK;
}

// ----------------------------------------------------------------------------------------
// Element kernels (submesh.cpp:66-160)
// ----------------------------------------------------------------------------------------
// Current-configuration Jacobian J = x dN and the gradient L = (dN J^-1)^T, 3 x npe.
inline void element_geometry(const Oracle& o, int e, int l, double* J, double* L) {
    const int npe = o.npe;
    const int* c = &o.conn[(size_t)e * npe];
    const double* dN = &o.sf.dN[(size_t)l * npe * 3];
    for (int i = 0; i < 9; ++i) J[i] = 0.0;
    for (int a = 0; a < npe; ++a) {
        const double* xa = &o.x[(size_t)c[a] * 3];
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; ++k) J[i * 3 + k] += xa[i] * dN[a * 3 + k];
    }
    double Ji[9];
    inv3(J, Ji);
    for (int a = 0; a < npe; ++a)
        for (int k = 0; k < 3; ++k)
            L[k * npe + a] = dN[a * 3 + 0] * Ji[0 * 3 + k] + dN[a * 3 + 1] * Ji[1 * 3 + k] +
                             dN[a * 3 + 2] * Ji[2 * 3 + k];
}

// tangent_stiffness = material_tangent_stiffness (:136-160) + geometric (:110-134)
void element_stiffness(const Oracle& o, int e, double* ke) {
    const int npe = o.npe, nd = 3 * npe, nq = o.nq;
    std::vector<double> kmat(nd * nd, 0.0), B(6 * nd, 0.0), BtD(nd * 6);
    for (int l = 0; l < nq; ++l) {
        double J[9], L[3 * 8];
        element_geometry(o, e, l, J, L);
        // symmetric_gradient<3> (gradient_operator.hpp:37-58)
        std::fill(B.begin(), B.end(), 0.0);
        for (int a = 0; a < npe; ++a) {
            int b = 3 * a;
            B[0 * nd + b] = L[0 * npe + a];
            B[4 * nd + b] = L[2 * npe + a];
            B[5 * nd + b] = L[1 * npe + a];
            B[1 * nd + b + 1] = L[1 * npe + a];
            B[3 * nd + b + 1] = L[2 * npe + a];
            B[5 * nd + b + 1] = L[0 * npe + a];
            B[2 * nd + b + 2] = L[2 * npe + a];
            B[3 * nd + b + 2] = L[1 * npe + a];
            B[4 * nd + b + 2] = L[0 * npe + a];
        }
        const double* D = &o.D[((size_t)e * nq + l) * 36];
        double detJ = det3(J);
        for (int i = 0; i < nd; ++i)
            for (int k = 0; k < 6; ++k) {
                double v = 0;
                for (int m = 0; m < 6; ++m) v += B[m * nd + i] * D[m * 6 + k];
                BtD[i * 6 + k] = v;
            }
        double w = o.sf.w[l];
        for (int i = 0; i < nd; ++i)
            for (int j = 0; j < nd; ++j) {
                double v = 0;
                for (int k = 0; k < 6; ++k) v += BtD[i * 6 + k] * B[k * nd + j];
                kmat[i * nd + j] += (v * detJ) * w;
            }
    }
    for (int i = 0; i < nd * nd; ++i) ke[i] = kmat[i];
    bool finite = (o.mat.model == NEO_HOOKE || o.mat.model == GAUSS_AFFINE_MICROSPHERE ||
                   o.mat.model == LANGEVIN_AFFINE_MICROSPHERE || o.mat.model == NONAFFINE_MICROSPHERE);
    if (!finite) return;
    std::vector<double> kgeo(npe * npe, 0.0);
    for (int l = 0; l < nq; ++l) {
        double J[9], L[3 * 8];
        element_geometry(o, e, l, J, L);
        const double* s = &o.sigma[((size_t)e * nq + l) * 9];
        double detJ = det3(J);
        double w = o.sf.w[l];
        for (int a = 0; a < npe; ++a) {
            double t[3];  // (L^T sigma) row a
            for (int k = 0; k < 3; ++k)
                t[k] = L[0 * npe + a] * s[0 * 3 + k] + L[1 * npe + a] * s[1 * 3 + k] +
                       L[2 * npe + a] * s[2 * 3 + k];
            for (int b = 0; b < npe; ++b) {
                double v = t[0] * L[0 * npe + b] + t[1] * L[1 * npe + b] + t[2] * L[2 * npe + b];
                kgeo[a * npe + b] += (v * detJ) * w;
            }
        }
    }
    // identity_expansion_inplace<3> (tensor_operations.hpp:121-135)
    for (int a = 0; a < npe; ++a)
        for (int b = 0; b < npe; ++b)
            for (int k = 0; k < 3; ++k) ke[(3 * a + k) * nd + 3 * b + k] += kgeo[a * npe + b];
}

// internal_force (submesh.cpp:82-108): f[a][j] += (sum_i L[i][a] sigma[i][j] detJ) w
void element_internal_force(const Oracle& o, int e, double* fe) {
    const int npe = o.npe, nq = o.nq;
    for (int i = 0; i < 3 * npe; ++i) fe[i] = 0.0;
    for (int l = 0; l < nq; ++l) {
        double J[9], L[3 * 8];
        element_geometry(o, e, l, J, L);
        const double* s = &o.sigma[((size_t)e * nq + l) * 9];
        double detJ = det3(J);
        double w = o.sf.w[l];
        for (int a = 0; a < npe; ++a)
            for (int j = 0; j < 3; ++j) {
                double v = 0;
                for (int i = 0; i < 3; ++i) v += L[i * npe + a] * s[i * 3 + j];
                fe[a * 3 + j] += (v * detJ) * w;
            }
    }
}

// add_to (thread_safe_plugin.hpp:7-23): binary search of the column in the row, atomic add
inline void add_to(Oracle& o, double* K, int row, int colv, double v) {
    const int* b = &o.col[o.rowptr[row]];
    const int* e = &o.col[o.rowptr[row + 1]];
    const int* p = std::lower_bound(b, e, colv);
    size_t idx = (size_t)(p - o.col.data());
#pragma omp atomic
    K[idx] += v;
}

// static_matrix::assemble_stiffness (static_matrix.hpp:243-277)
void assemble_stiffness(Oracle& o, double* K) {
    std::fill(K, K + o.col.size(), 0.0);
    const int npe = o.npe, nd = 3 * npe;
#pragma omp parallel
    {
        std::vector<double> ke(nd * nd);
#pragma omp for schedule(dynamic, 64)
        for (int e = 0; e < o.E; ++e) {
            element_stiffness(o, e, ke.data());
            const int* c = &o.conn[(size_t)e * npe];
            for (int b = 0; b < nd; ++b)
                for (int a = 0; a < nd; ++a)
                    add_to(o, K, 3 * c[a / 3] + a % 3, 3 * c[b / 3] + b % 3, ke[a * nd + b]);
        }
    }
}

// static_matrix::compute_internal_force (static_matrix.hpp:189-203), serial
void compute_internal_force(const Oracle& o, double* f) {
    std::fill(f, f + 3 * o.N, 0.0);
    const int npe = o.npe;
    double fe[24];
    for (int e = 0; e < o.E; ++e) {
        element_internal_force(o, e, fe);
        const int* c = &o.conn[(size_t)e * npe];
        for (int a = 0; a < npe; ++a)
            for (int j = 0; j < 3; ++j) f[3 * c[a] + j] += fe[a * 3 + j];
    }
}

// internal_variables::commit / revert (internal_variables.hpp:202-214)
void save_internal_variables(Oracle& o, bool converged) {
    if (converged) {
        o.ep_old = o.ep;
        o.epbar_old = o.epbar;
        o.sigma_old = o.sigma;
        o.F_old = o.F;
    } else {
        o.ep = o.ep_old;
        o.epbar = o.epbar_old;
        o.sigma = o.sigma_old;
        o.F = o.F_old;
    }
}

// ----------------------------------------------------------------------------------------
// Linear solver: conjugate_gradient::solve (linear_solver.cpp:67-109) = RCM (computed once)
// + P^T A P + Eigen ConjugateGradient<Lower|Upper> with the diagonal preconditioner.
// ----------------------------------------------------------------------------------------
struct Csr {
    int n = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
};

// graph/cuthill_mckee.hpp:11-97 + graph/adjacency_graph.hpp:10-71
std::vector<int> reverse_cuthill_mckee(int n, const int* rp, const int* ci) {
    std::vector<std::vector<int>> adj(n);
    for (int i = 0; i < n; ++i) {
        for (int p = rp[i]; p < rp[i + 1]; ++p) adj[i].push_back(ci[p]);
        auto it = std::find(adj[i].begin(), adj[i].end(), i);
        if (it != adj[i].end()) adj[i].erase(it);
    }
    // minimum_degree_sort: std::sort of each adjacency list by neighbour degree
    for (auto& a : adj)
        std::sort(a.begin(), a.end(), [&](int l, int r) { return adj[l].size() < adj[r].size(); });
    std::vector<int> perm;
    perm.reserve(n);
    std::vector<bool> done(n, false);
    std::queue<int> queue;
    auto push_children = [&](int node) {
        for (int c : adj[node])
            if (!done[c]) queue.push(c);
    };
    while ((int)perm.size() != n) {
        // find_lowest_degree: first lowest-degree node not yet reordered
        int count = n, node = n;
        for (int r = 0; r < n; ++r) {
            int d = (int)adj[r].size();
            if (d < count && !done[r]) {
                count = d;
                node = r;
            }
        }
        perm.push_back(node);
        done[node] = true;
        push_children(node);
        while (!queue.empty()) {
            int f = queue.front();
            if (!done[f]) {
                done[f] = true;
                perm.push_back(f);
                push_children(f);
            }
            queue.pop();
        }
    }
    std::reverse(perm.begin(), perm.end());
    return perm;
}

// A' = P^T A P with new index i <-> old index perm[i]; columns sorted per row.
void permute_symmetric(const Csr& A, const std::vector<int>& perm, Csr& out) {
    int n = A.n;
    std::vector<int> inv(n);
    for (int i = 0; i < n; ++i) inv[perm[i]] = i;
    out.n = n;
    out.rp.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) out.rp[i + 1] = out.rp[i] + (A.rp[perm[i] + 1] - A.rp[perm[i]]);
    out.ci.resize(A.ci.size());
    out.v.resize(A.v.size());
    std::vector<std::pair<int, double>> row;
    for (int i = 0; i < n; ++i) {
        int o = perm[i];
        row.clear();
        for (int p = A.rp[o]; p < A.rp[o + 1]; ++p) row.emplace_back(inv[A.ci[p]], A.v[p]);
        std::sort(row.begin(), row.end(),
                  [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
                      return a.first < b.first;
                  });
        int q = out.rp[i];
        for (auto& pr : row) {
            out.ci[q] = pr.first;
            out.v[q] = pr.second;
            ++q;
        }
    }
}

inline double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// Eigen's row-major sparse * dense product (parallel over rows)
void spmv(const Csr& A, const std::vector<double>& x, std::vector<double>& y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < A.n; ++i) {
        double s = 0.0;
        for (int p = A.rp[i]; p < A.rp[i + 1]; ++p) s += A.v[p] * x[A.ci[p]];
        y[i] = s;
    }
}

// The published PCG algorithm as Eigen's internal::conjugate_gradient states it.
void eigen_pcg(const Csr& A, const std::vector<double>& b, std::vector<double>& x, double tol,
               int maxit, int& iters, double& error) {
    int n = A.n;
    x.assign(n, 0.0);
    std::vector<double> invdiag(n, 1.0);
    for (int i = 0; i < n; ++i)
        for (int p = A.rp[i]; p < A.rp[i + 1]; ++p)
            if (A.ci[p] == i) {
                if (A.v[p] != 0.0) invdiag[i] = 1.0 / A.v[p];
                break;
            }
    std::vector<double> r(b), p(n), z(n), tmp(n);
    double rhsNorm2 = dot(b, b);
    if (rhsNorm2 == 0) {
        x.assign(n, 0.0);
        iters = 0;
        error = 0;
        return;
    }
    double threshold = std::max(tol * tol * rhsNorm2, std::numeric_limits<double>::min());
    double residualNorm2 = dot(r, r);
    if (residualNorm2 < threshold) {
        iters = 0;
        error = std::sqrt(residualNorm2 / rhsNorm2);
        return;
    }
    for (int i = 0; i < n; ++i) p[i] = invdiag[i] * r[i];
    double absNew = dot(r, p);
    int i = 0;
    while (i < maxit) {
        spmv(A, p, tmp);
        double alpha = absNew / dot(p, tmp);
        for (int k = 0; k < n; ++k) x[k] += alpha * p[k];
        for (int k = 0; k < n; ++k) r[k] -= alpha * tmp[k];
        residualNorm2 = dot(r, r);
        if (residualNorm2 < threshold) break;
        for (int k = 0; k < n; ++k) z[k] = invdiag[k] * r[k];
        double absOld = absNew;
        absNew = dot(r, z);
        double beta = absNew / absOld;
        for (int k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
        ++i;
    }
    error = std::sqrt(residualNorm2 / rhsNorm2);
    iters = i;
}

struct CgSolver {
    double tol = 1e-5;
    int maxit = 2000;
    bool use_rcm = true;
    bool have_perm = false;
    std::vector<int> perm;
    long long total_iterations = 0;
    int last_iterations = 0;
    double last_error = 0;

    int solve(const Csr& A, std::vector<double>& x, const std::vector<double>& b) {
        int n = A.n;
        int it = 0;
        double err = 0;
        if (use_rcm) {
            if (!have_perm) {
                perm = reverse_cuthill_mckee(n, A.rp.data(), A.ci.data());
                have_perm = true;
            }
            Csr Ap;
            permute_symmetric(A, perm, Ap);
            std::vector<double> bp(n), xp;
            for (int i = 0; i < n; ++i) bp[i] = b[perm[i]];
            eigen_pcg(Ap, bp, xp, tol, maxit, it, err);
            x.assign(n, 0.0);
            for (int i = 0; i < n; ++i) x[perm[i]] = xp[i];
        } else {
            eigen_pcg(A, b, x, tol, maxit, it, err);
        }
        last_iterations = it;
        last_error = err;
        total_iterations += it;
        for (double v : x)
            if (std::isnan(v)) return ORC_E_NAN;
        if (it >= maxit) return ORC_E_CG_MAXIT;
        return ORC_OK;
    }
};

// ----------------------------------------------------------------------------------------
// Boundary values and adaptive load stepping
// ----------------------------------------------------------------------------------------
struct TimeTable {
    std::vector<double> t, v;
    // boundary.cpp:55-85: exact time match (is_approx, relative 1e-10) else linear interpolation
    double value(double time) const {
        for (size_t i = 0; i < t.size(); ++i) {
            double a = t[i], b = time;
            bool match;
            {
                double maxv = std::numeric_limits<double>::max(),
                       minv = std::numeric_limits<double>::min();
                double rd;
                if (std::isnan(a) || std::isnan(b))
                    rd = maxv;
                else if (((a < 0) != (b < 0)) && a != 0 && b != 0)
                    rd = maxv;
                else {
                    double x1 = std::fabs(a), y1 = std::fabs(b);
                    if (x1 < minv) x1 = minv;
                    if (y1 < minv) y1 = minv;
                    rd = std::max(std::fabs((x1 - y1) / x1), std::fabs((x1 - y1) / y1));
                }
                match = rd <= 1e-10 || std::fabs(a - b) <= 0.0;
            }
            if (match) return v[i];
        }
        for (size_t i = 0; i + 1 < t.size(); ++i)
            if (t[i] < time && time < t[i + 1]) {
                double f = (time - t[i]) / (t[i + 1] - t[i]);
                return (1.0 - f) * v[i] + f * v[i + 1];
            }
        return v.back();
    }
    bool active(double time) const { return time >= t.front() && time <= t.back(); }
};

struct DofBoundary {
    std::vector<int> dofs;
    std::vector<double> weights;  // nodal forces only: f_ext[dof] += weight * value(t)
    TimeTable table;
};

// solver/adaptive_time_step.cpp:12-165
struct AdaptiveTimeStep {
    int increment_limit = 5;
    int successful_increments = 0, consecutive_converged = 0, consecutive_unconverged = 0;
    double initial_time = 1.0, final_time = 1.0, current_time = 1.0, total_time = 0.0;
    double last_converged_time = 0.0, last_converged_time_step_size = 0.0;
    double minimum_increment = 0, maximum_increment = 0;
    bool is_applied = false;
    std::priority_queue<double, std::vector<double>, std::greater<double>> queue;

    void init(double period, double initial, double minimum, double maximum, bool adaptive,
              const std::vector<double>& history) {
        for (double t : history) queue.push(t);
        if (!queue.empty() && is_approx_zero(queue.top(), 0.0)) queue.pop();
        initial_time = initial;
        minimum_increment = adaptive ? minimum : initial;
        maximum_increment = adaptive ? maximum : initial;
        final_time = period;
        current_time = std::min(queue.empty() ? initial : queue.top(), initial_time);
    }
    double step_time() const { return current_time; }
    double increment() const { return current_time - last_converged_time; }
    bool highly_nonlinear() const { return consecutive_unconverged > 0 || consecutive_converged < 4; }
    // returns ORC_OK, or ORC_E_CUTBACK_LIMIT when the reference throws std::domain_error
    int update(bool converged) {
        if (converged) {
            if (!queue.empty() && current_time >= queue.top()) queue.pop();
            last_converged_time_step_size = current_time - last_converged_time;
            last_converged_time = current_time;
            double d = current_time - final_time;
            bool eq;
            {
                double a = current_time, b = final_time;
                double maxv = std::numeric_limits<double>::max(),
                       minv = std::numeric_limits<double>::min();
                double rd;
                if (((a < 0) != (b < 0)) && a != 0 && b != 0)
                    rd = maxv;
                else {
                    double x1 = std::fabs(a), y1 = std::fabs(b);
                    if (x1 < minv) x1 = minv;
                    if (y1 < minv) y1 = minv;
                    rd = std::max(std::fabs((x1 - y1) / x1), std::fabs((x1 - y1) / y1));
                }
                eq = rd <= 1e-10 || std::fabs(d) <= 0.0;
            }
            is_applied = eq || queue.empty();
            consecutive_unconverged = 0;
            consecutive_converged++;
            successful_increments++;
            if (is_applied) return ORC_OK;
            double new_time = std::min(highly_nonlinear()
                                           ? last_converged_time_step_size + current_time
                                           : 2.0 * current_time,
                                       current_time + maximum_increment);
            current_time = std::min(queue.top(), std::min(new_time, final_time));
            return ORC_OK;
        }
        double dt = std::max(minimum_increment, (current_time - last_converged_time) * 0.5);
        current_time = last_converged_time + dt;
        if (current_time > final_time) return ORC_E_CUTBACK_LIMIT;
        consecutive_unconverged++;
        consecutive_converged = 0;
        if (consecutive_unconverged == increment_limit) return ORC_E_CUTBACK_LIMIT;
        return ORC_OK;
    }
};

// ----------------------------------------------------------------------------------------
// static_matrix (static_matrix.hpp:29-467)
// ----------------------------------------------------------------------------------------
struct NewtonLog {
    double step_time;
    int iteration;
    int cg_iterations;
    double displacement_norm, force_norm;
};

struct StaticMatrix {
    Oracle* o = nullptr;
    std::vector<DofBoundary> dirichlet;  // in the reference's iteration order
    std::vector<DofBoundary> nodal_forces;
    AdaptiveTimeStep load;
    CgSolver solver;
    bool use_relative_norm = true;
    double residual_tolerance = 1e-3, displacement_tolerance = 1e-3;
    int maximum_iterations = 10;
    double norm_initial_residual = 1.0, displacement_norm = 0, force_norm = 0;
    Csr Kt;
    std::vector<double> f_int, f_ext, u, u_old, delta_d, minus_residual;
    std::vector<NewtonLog> log;
    std::string message;
    long long newton_iterations = 0;
    double seconds_assembly = 0, seconds_update = 0, seconds_solve = 0;

    void compute_external_force() {
        std::fill(f_ext.begin(), f_ext.end(), 0.0);
        double t = load.step_time();
        for (auto& b : nodal_forces) {
            double v = b.table.value(t);
            for (size_t i = 0; i < b.dofs.size(); ++i)
                f_ext[b.dofs[i]] += (b.weights.empty() ? 1.0 : b.weights[i]) * v;
        }
    }

    void apply_displacement_boundaries() {
        // sparse increment, later boundaries overwrite earlier ones (coeffRef assignment)
        int n = o->ndofs();
        std::vector<double> inc(n, 0.0);
        std::vector<char> set(n, 0);
        for (auto& b : dirichlet) {
            if (!b.table.active(load.step_time())) continue;
            double du = b.table.value(load.step_time()) - b.table.value(load.last_converged_time);
            for (int d : b.dofs) {
                inc[d] = du;
                set[d] = 1;
            }
        }
        std::vector<double> Kinc(n);
        spmv(Kt, inc, Kinc);
        for (int i = 0; i < n; ++i) minus_residual[i] -= Kinc[i];
        for (int i = 0; i < n; ++i)
            if (set[i]) u[i] += inc[i];
    }

    void enforce_dirichlet_conditions(Csr& A, std::vector<double>& b) {
        for (auto& bc : dirichlet) {
            if (!bc.table.active(load.step_time())) continue;
            for (int d : bc.dofs) {
                double diag = 0.0;
                for (int p = A.rp[d]; p < A.rp[d + 1]; ++p)
                    if (A.ci[p] == d) diag = A.v[p];
                b[d] = 0.0;
                for (int p = A.rp[d]; p < A.rp[d + 1]; ++p) {
                    A.v[p] = 0.0;
                    int c = A.ci[p];
                    int* s = &A.ci[A.rp[c]];
                    int* e = &A.ci[A.rp[c + 1]];
                    int* q = std::lower_bound(s, e, d);
                    A.v[q - A.ci.data()] = 0.0;
                }
                for (int p = A.rp[d]; p < A.rp[d + 1]; ++p)
                    if (A.ci[p] == d) A.v[p] = diag;
            }
        }
    }

    static double norm(const std::vector<double>& v) { return std::sqrt(dot(v, v)); }

    void update_relative_norms() {
        double un = norm(u), fe = norm(f_ext), fi = norm(f_int);
        if (use_relative_norm && !is_approx_zero(un, 1.0) &&
            !is_approx_zero(std::max(fe, fi), 1.0)) {
            displacement_norm = norm(delta_d) / un;
            force_norm = norm(minus_residual) / std::max(norm_initial_residual, std::max(fe, fi));
        } else {
            displacement_norm = norm(delta_d);
            force_norm = norm(minus_residual);
        }
    }

    // perform_equilibrium_iterations (:402-467).  Returns OK or a recoverable error.
    int equilibrium() {
        int n = o->ndofs();
        u = u_old;
        int st = update_internal_variables(*o, u.data(), &message);
        if (st) return st;
        int k = 0;
        while (k < maximum_iterations) {
            double t0 = wtime();
            assemble_stiffness(*o, Kt.v.data());
            double t1 = wtime();
            seconds_assembly += t1 - t0;
            compute_internal_force(*o, f_int.data());
            for (int i = 0; i < n; ++i) minus_residual[i] = f_ext[i] - f_int[i];
            if (k == 0) {
                apply_displacement_boundaries();
                norm_initial_residual = norm(minus_residual);
            }
            enforce_dirichlet_conditions(Kt, minus_residual);
            double t2 = wtime();
            st = solver.solve(Kt, delta_d, minus_residual);
            seconds_solve += wtime() - t2;
            if (st) {
                message = "Conjugate gradient solver maximum iterations reached";
                return st;
            }
            for (int i = 0; i < n; ++i) u[i] += delta_d[i];
            double t3 = wtime();
            st = update_internal_variables(*o, u.data(), &message);
            seconds_update += wtime() - t3;
            if (st) return st;
            update_relative_norms();
            log.push_back({load.step_time(), k, solver.last_iterations, displacement_norm, force_norm});
            ++newton_iterations;
            if (displacement_norm <= displacement_tolerance && force_norm <= residual_tolerance) break;
            ++k;
        }
        if (k == maximum_iterations) {
            message = "Reached Newton-Raphson iteration limit";
            return ORC_E_NEWTON_MAXIT;
        }
        u_old = u;
        int s2 = load.update(true);
        save_internal_variables(*o, true);
        return s2 == ORC_OK ? ORC_OK : -s2;  // negative: non-recoverable
    }

    // solve (:145-187); the recursion on computational_error is an explicit loop.
    int solve() {
        int n = o->ndofs();
        f_int.assign(n, 0.0);
        f_ext.assign(n, 0.0);
        u.assign(n, 0.0);
        u_old.assign(n, 0.0);
        delta_d.assign(n, 0.0);
        minus_residual.assign(n, 0.0);
        Kt.n = n;
        Kt.rp = o->rowptr;
        Kt.ci = o->col;
        Kt.v.assign(o->col.size(), 0.0);
        for (;;) {
            // mesh.update_internal_variables(displacement) inside the same try block
            int st = update_internal_variables(*o, u.data(), &message);
            bool failed = st != ORC_OK;
            while (!failed && !load.is_applied) {
                compute_external_force();
                st = equilibrium();
                if (st < 0) return -st;
                if (st != ORC_OK) {
                    failed = true;
                    break;
                }
            }
            if (!failed) return ORC_OK;
            if (load.update(false) != ORC_OK) return ORC_E_CUTBACK_LIMIT;
            save_internal_variables(*o, false);
            u = u_old;
        }
    }
};

// Non-follower loads per unit load value (the load's time table scales them), in the initial
// configuration, accumulated into f [3N] in element order.  Surface groups (quad4 or tri3 faces
// of the boundary mesh, neon local node order):
//   traction  f[3a+k] += sum_q w N_a |X,xi x X,eta|            (neumann.hpp:69-133, traction.hpp)
//   pressure  f[3a+i] += -sum_q w N_a n_i |X,xi x X,eta|, n = (X,xi x X,eta)/|..|
//             (pressure.cpp:9-37: positive pressure compresses the surface)
// with quadrilateral4 (interpolations/quadrilateral.cpp:17-45) on the 4-point or, reduced, the
// 1-point rule (quadrilateral_quadrature.cpp:5-24), triangle3 (interpolations/triangle.cpp:16-40)
// on its 1-point rule (triangle_quadrature.cpp:12-16, weights x 0.5), chosen as
// make_surface_interpolation does (interpolation_factory.cpp:99-117).  Volume group (the mesh's
// own elements):
//   body force f[3a+k] += sum_q w N_a det(X dN)                (neumann.hpp:135-192, body_force.hpp)
// kind: 0 traction, 1 pressure, 2 body force; k = component (traction, body force).
void nonfollower_load(const Oracle& o, int kind, int component, const int* faces, int nfaces,
                      int npf, int reduced, double* f) {
    if (kind == 2) {
        // the volume interpolation: hex8 8-point or tet4 1-point, N at the points
        const int nq = o.sf.nq, npe = o.npe;
        std::vector<double> N((size_t)nq * npe);
        if (npe == 8) {
            const double lc[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                     {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
            const double g = 1.0 / std::sqrt(3.0);
            for (int l = 0; l < nq; ++l)
                for (int a = 0; a < npe; ++a)
                    N[l * npe + a] = 1.0 / 8.0 * (1.0 + lc[a][0] * lc[l][0] * g) *
                                     (1.0 + lc[a][1] * lc[l][1] * g) *
                                     (1.0 + lc[a][2] * lc[l][2] * g);
        } else {
            for (int a = 0; a < 4; ++a) N[a] = 0.25;  // (r, s, t, 1-r-s-t) at (1/4, 1/4, 1/4)
        }
        for (int e = 0; e < o.E; ++e) {
            const int* c = &o.conn[(size_t)e * npe];
            std::vector<double> fe(npe, 0.0);
            for (int l = 0; l < nq; ++l) {
                double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                for (int a = 0; a < npe; ++a)
                    for (int i = 0; i < 3; ++i)
                        for (int k = 0; k < 3; ++k)
                            J[i * 3 + k] += o.X[3 * (size_t)c[a] + i] * o.sf.dN[(l * npe + a) * 3 + k];
                const double j = det3(J);
                for (int a = 0; a < npe; ++a) fe[a] += N[l * npe + a] * j * o.sf.w[l];
            }
            for (int a = 0; a < npe; ++a) f[3 * (size_t)c[a] + component] += fe[a];
        }
        return;
    }
    // surface interpolation
    std::vector<double> qxi, qeta, qw;
    if (npf == 4) {
        const double g = 1.0 / std::sqrt(3.0);
        if (reduced) {
            qxi = {0.0}; qeta = {0.0}; qw = {4.0};
        } else {
            qxi = {-g, g, g, -g}; qeta = {-g, -g, g, g}; qw = {1.0, 1.0, 1.0, 1.0};
        }
    } else {
        qxi = {1.0 / 3.0}; qeta = {1.0 / 3.0}; qw = {0.5};
    }
    const double lq[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    for (int fc = 0; fc < nfaces; ++fc) {
        const int* c = &faces[(size_t)fc * npf];
        double fe[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (size_t l = 0; l < qw.size(); ++l) {
            double N[4], r[4][2];
            if (npf == 4) {
                for (int a = 0; a < 4; ++a) {
                    N[a] = 0.25 * (1.0 + lq[a][0] * qxi[l]) * (1.0 + lq[a][1] * qeta[l]);
                    r[a][0] = 0.25 * (1.0 + lq[a][1] * qeta[l]) * lq[a][0];
                    r[a][1] = 0.25 * (1.0 + lq[a][0] * qxi[l]) * lq[a][1];
                }
            } else {
                N[0] = qxi[l]; N[1] = qeta[l]; N[2] = 1.0 - qxi[l] - qeta[l];
                r[0][0] = 1.0; r[0][1] = 0.0; r[1][0] = 0.0; r[1][1] = 1.0;
                r[2][0] = -1.0; r[2][1] = -1.0;
            }
            double t0[3] = {0, 0, 0}, t1[3] = {0, 0, 0};  // the columns of the 3x2 Jacobian
            for (int a = 0; a < npf; ++a)
                for (int i = 0; i < 3; ++i) {
                    t0[i] += o.X[3 * (size_t)c[a] + i] * r[a][0];
                    t1[i] += o.X[3 * (size_t)c[a] + i] * r[a][1];
                }
            const double cr[3] = {t0[1] * t1[2] - t0[2] * t1[1], t0[2] * t1[0] - t0[0] * t1[2],
                                  t0[0] * t1[1] - t0[1] * t1[0]};
            const double j = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
            for (int a = 0; a < npf; ++a) {
                if (kind == 0) {
                    fe[a][component] += N[a] * j * qw[l];
                } else {
                    for (int i = 0; i < 3; ++i) fe[a][i] += N[a] * (cr[i] / j) * j * qw[l];
                }
            }
        }
        for (int a = 0; a < npf; ++a)
            for (int i = 0; i < 3; ++i)
                f[3 * (size_t)c[a] + i] += (kind == 1 ? -fe[a][i] : fe[a][i]);
    }
}

}  // namespace

// ========================================================================================
// C-ABI (ctypes) -- test / baseline harness only
// ========================================================================================
extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// params: [K, G, sigma_y, H_iso, segments_per_chain]
void* orc_create(int num_nodes, const double* coords, int num_elements, int nodes_per_element,
                 const int* conn, int model, const double* params, const double* Ge) {
    if (nodes_per_element != 8 && nodes_per_element != 4) return nullptr;
    auto* o = new Oracle();
    o->N = num_nodes;
    o->E = num_elements;
    o->npe = nodes_per_element;
    o->sf = nodes_per_element == 8 ? make_hex8() : make_tet4();
    o->nq = o->sf.nq;
    o->X.assign(coords, coords + 3 * (size_t)num_nodes);
    o->x = o->X;
    o->conn.assign(conn, conn + (size_t)num_elements * nodes_per_element);
    o->mat.model = model;
    o->mat.K = params[0];
    o->mat.G = params[1];
    o->mat.sigma_y = params[2];
    o->mat.H_iso = params[3];
    o->mat.segments = params[4];
    o->mat.nonaffine_p = params[5];
    o->mat.sphere_points = params[6] == 33.0 ? 33 : 21;
    o->sphere = o->mat.sphere_points == 33 ? make_bo33() : make_bo21();
    if (Ge) o->Ge.assign(Ge, Ge + num_elements);
    size_t nqp = (size_t)num_elements * o->nq;
    o->H.assign(nqp * 9, 0.0);
    o->F.assign(nqp * 9, 0.0);
    for (size_t q = 0; q < nqp; ++q) o->F[q * 9 + 0] = o->F[q * 9 + 4] = o->F[q * 9 + 8] = 1.0;
    o->detF.assign(nqp, 1.0);
    o->sigma.assign(nqp * 9, 0.0);
    o->D.assign(nqp * 36, 0.0);
    o->vm.assign(nqp, 0.0);
    o->ep.assign(nqp * 9, 0.0);
    o->epbar.assign(nqp, 0.0);
    if (model == LINEAR_ELASTIC || model == J2_SMALL_STRAIN)
        for (size_t q = 0; q < nqp; ++q) isotropic_voigt(o->mat.lambda(), o->mat.G, &o->D[q * 36]);
    save_internal_variables(*o, true);
    build_pattern(*o);
    return o;
}

void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }

// directions [n][3] and weights [n] of the BO21 (points 21) or BO33 (points 33) rule; returns n
int orc_sphere_rule(int points, double* r, double* w) {
    SphereRule s = points == 33 ? make_bo33() : make_bo21();
    for (int i = 0; i < s.n; ++i) {
        for (int k = 0; k < 3; ++k) r[3 * i + k] = s.r[i][k];
        w[i] = s.w[i];
    }
    return s.n;
}

// hex8 (npe 8) or tet4 (npe 4) shape derivatives [nq][npe][3] and weights [nq]
int orc_shape(int npe, double* dN, double* w) {
    Interpolation I = npe == 8 ? make_hex8() : make_tet4();
    std::copy(I.dN.begin(), I.dN.end(), dN);
    std::copy(I.w.begin(), I.w.end(), w);
    return I.nq;
}
int orc_ndofs(void* h) { return static_cast<Oracle*>(h)->ndofs(); }
long long orc_nnz(void* h) { return static_cast<Oracle*>(h)->nnz(); }

void orc_pattern(void* h, int* rowptr, int* col) {
    auto* o = static_cast<Oracle*>(h);
    std::copy(o->rowptr.begin(), o->rowptr.end(), rowptr);
    std::copy(o->col.begin(), o->col.end(), col);
}

int orc_update(void* h, const double* u, char* msg, int msglen) {
    auto* o = static_cast<Oracle*>(h);
    std::string m;
    int st = update_internal_variables(*o, u, &m);
    if (msg && msglen > 0) std::snprintf(msg, msglen, "%s", m.c_str());
    return st;
}

void orc_assemble(void* h, double* K) { assemble_stiffness(*static_cast<Oracle*>(h), K); }
void orc_internal_force(void* h, double* f) { compute_internal_force(*static_cast<Oracle*>(h), f); }
void orc_element_stiffness(void* h, int e, double* ke) {
    element_stiffness(*static_cast<Oracle*>(h), e, ke);
}
void orc_save(void* h, int converged) { save_internal_variables(*static_cast<Oracle*>(h), converged); }

// which: 0 sigma(9/qp) 1 D(36/qp) 2 detF(1/qp) 3 ep(9/qp) 4 epbar(1/qp) 5 vm 6 F(9/qp) 7 H(9/qp)
void orc_get_qp(void* h, int which, double* out) {
    auto* o = static_cast<Oracle*>(h);
    const std::vector<double>* v = nullptr;
    switch (which) {
        case 0: v = &o->sigma; break;
        case 1: v = &o->D; break;
        case 2: v = &o->detF; break;
        case 3: v = &o->ep; break;
        case 4: v = &o->epbar; break;
        case 5: v = &o->vm; break;
        case 6: v = &o->F; break;
        case 7: v = &o->H; break;
        default: return;
    }
    std::copy(v->begin(), v->end(), out);
}

void orc_set_qp(void* h, int which, const double* in) {
    auto* o = static_cast<Oracle*>(h);
    std::vector<double>* v = nullptr;
    switch (which) {
        case 0: v = &o->sigma; break;
        case 1: v = &o->D; break;
        case 2: v = &o->detF; break;
        case 3: v = &o->ep; break;
        case 4: v = &o->epbar; break;
        case 6: v = &o->F; break;
        case 7: v = &o->H; break;
        default: return;
    }
    std::copy(in, in + v->size(), v->begin());
}

// Constitutive update only, on inputs already placed with orc_set_qp (H, F, detF): the
// single-point model checks of test/small_strain_constitutive.cpp and
// test/hyperelastic_constitutive.cpp.
int orc_constitutive_only(void* h) {
    auto* o = static_cast<Oracle*>(h);
    size_t nqp = (size_t)o->E * o->nq;
    for (size_t q = 0; q < nqp; ++q) {
        switch (o->mat.model) {
            case LINEAR_ELASTIC: update_linear_elastic(*o, q); break;
            case NEO_HOOKE: update_neo_hooke(*o, q); break;
            case J2_SMALL_STRAIN:
                if (update_j2(*o, q)) return ORC_E_RETURN_MAP;
                break;
            case GAUSS_AFFINE_MICROSPHERE: update_microsphere(*o, q, o->shear((int)(q / o->nq))); break;
            case LANGEVIN_AFFINE_MICROSPHERE:
                update_microsphere(*o, q, o->shear((int)(q / o->nq)), true);
                break;
            case NONAFFINE_MICROSPHERE: update_nonaffine(*o, q, o->shear((int)(q / o->nq))); break;
        }
    }
    return ORC_OK;
}

// conjugate_gradient::solve on a caller CSR (test/linear_solvers.cpp drives the same call)
int orc_cg_solve(int n, const int* rowptr, const int* col, const double* val, const double* b,
                 double* x, double tol, int maxit, int use_rcm, int* iters, double* err) {
    Csr A;
    A.n = n;
    A.rp.assign(rowptr, rowptr + n + 1);
    A.ci.assign(col, col + rowptr[n]);
    A.v.assign(val, val + rowptr[n]);
    CgSolver s;
    s.tol = tol;
    s.maxit = maxit;
    s.use_rcm = use_rcm != 0;
    std::vector<double> bb(b, b + n), xx;
    int st = s.solve(A, xx, bb);
    std::copy(xx.begin(), xx.end(), x);
    if (iters) *iters = s.last_iterations;
    if (err) *err = s.last_error;
    return st;
}

// Time a bounded number of PCG iterations of the reference algorithm (CPU baseline sample):
// the per-solve P^T A P rebuild plus `iterations` CG iterations.  Returns the seconds spent.
double orc_cg_sample(int n, const int* rowptr, const int* col, const double* val, const double* b,
                     int iterations, int use_rcm, double* seconds_permute) {
    Csr A;
    A.n = n;
    A.rp.assign(rowptr, rowptr + n + 1);
    A.ci.assign(col, col + rowptr[n]);
    A.v.assign(val, val + rowptr[n]);
    std::vector<double> bb(b, b + n), x;
    double t0 = wtime();
    Csr Ap;
    const Csr* M = &A;
    std::vector<double> bp = bb;
    if (use_rcm) {
        std::vector<int> perm = reverse_cuthill_mckee(n, A.rp.data(), A.ci.data());
        double tp = wtime();
        permute_symmetric(A, perm, Ap);
        for (int i = 0; i < n; ++i) bp[i] = bb[perm[i]];
        if (seconds_permute) *seconds_permute = wtime() - tp;
        M = &Ap;
    }
    double t1 = wtime();
    int it;
    double err;
    eigen_pcg(*M, bp, x, 0.0, iterations, it, err);
    (void)t0;
    return wtime() - t1;
}

struct orc_options {
    double residual_tolerance, displacement_tolerance;
    int linear_iterations;  // maximum Newton iterations
    int absolute_tolerance;
    double period, initial, minimum, maximum;
    int adaptive;
    double cg_tolerance;
    int cg_maximum_iterations;
    int use_rcm;
};

struct orc_report {
    int status;
    int load_steps;
    long long newton_iterations;
    long long cg_iterations;
    double seconds_assembly, seconds_update, seconds_solve;
    char message[256];
};

// Dirichlet / nodal-force tables in the reference's iteration order:
// bc_dof_off[nbc+1] into bc_dofs, bc_pt_off[nbc+1] into bc_t / bc_v; nf_w (nullable) holds a
// per-DOF weight of each nodal-force table (consistent forces of a unit traction).
// log_out: [max_log][5] = (step_time, iteration, cg_iterations, disp_norm, force_norm)
int orc_static_solve(void* h, const orc_options* opt, int nbc, const int* bc_dof_off,
                     const int* bc_dofs, const int* bc_pt_off, const double* bc_t,
                     const double* bc_v, int nnf, const int* nf_dof_off, const int* nf_dofs,
                     const int* nf_pt_off, const double* nf_t, const double* nf_v,
                     const double* nf_w, double* u_out,
                     double* f_int_out, orc_report* rep, double* log_out, int max_log) {
    auto* o = static_cast<Oracle*>(h);
    StaticMatrix sm;
    sm.o = o;
    sm.residual_tolerance = opt->residual_tolerance;
    sm.displacement_tolerance = opt->displacement_tolerance;
    sm.maximum_iterations = opt->linear_iterations;
    sm.use_relative_norm = opt->absolute_tolerance == 0;
    sm.solver.tol = opt->cg_tolerance;
    sm.solver.maxit = opt->cg_maximum_iterations;
    sm.solver.use_rcm = opt->use_rcm != 0;
    std::vector<double> history;
    auto read = [&](int nb, const int* doff, const int* dofs, const int* poff, const double* t,
                    const double* v, std::vector<DofBoundary>& out) {
        for (int b = 0; b < nb; ++b) {
            DofBoundary d;
            d.dofs.assign(dofs + doff[b], dofs + doff[b + 1]);
            d.table.t.assign(t + poff[b], t + poff[b + 1]);
            d.table.v.assign(v + poff[b], v + poff[b + 1]);
            history.insert(history.end(), d.table.t.begin(), d.table.t.end());
            out.push_back(std::move(d));
        }
    };
    read(nbc, bc_dof_off, bc_dofs, bc_pt_off, bc_t, bc_v, sm.dirichlet);
    read(nnf, nf_dof_off, nf_dofs, nf_pt_off, nf_t, nf_v, sm.nodal_forces);
    if (nf_w)
        for (int b = 0; b < nnf; ++b)
            sm.nodal_forces[b].weights.assign(nf_w + nf_dof_off[b], nf_w + nf_dof_off[b + 1]);
    std::sort(history.begin(), history.end());
    history.erase(std::unique(history.begin(), history.end()), history.end());
    if (history.empty()) history = {0.0, opt->period};
    sm.load.init(opt->period, opt->initial, opt->minimum, opt->maximum, opt->adaptive != 0, history);
    int st = sm.solve();
    if (u_out) std::copy(sm.u.begin(), sm.u.end(), u_out);
    if (f_int_out) std::copy(sm.f_int.begin(), sm.f_int.end(), f_int_out);
    if (rep) {
        rep->status = st;
        rep->load_steps = sm.load.successful_increments;
        rep->newton_iterations = sm.newton_iterations;
        rep->cg_iterations = sm.solver.total_iterations;
        rep->seconds_assembly = sm.seconds_assembly;
        rep->seconds_update = sm.seconds_update;
        rep->seconds_solve = sm.seconds_solve;
        std::snprintf(rep->message, sizeof rep->message, "%s", sm.message.c_str());
    }
    if (log_out)
        for (int i = 0; i < (int)sm.log.size() && i < max_log; ++i) {
            log_out[i * 5 + 0] = sm.log[i].step_time;
            log_out[i * 5 + 1] = sm.log[i].iteration;
            log_out[i * 5 + 2] = sm.log[i].cg_iterations;
            log_out[i * 5 + 3] = sm.log[i].displacement_norm;
            log_out[i * 5 + 4] = sm.log[i].force_norm;
        }
    return st;
}

// shape_function::compute_extrapolation_matrix (interpolations/shape_function.hpp:70-100) for the
// two element types of the path.  hex8 with its 8 points: m == n, E = N^-1 where row l of N holds
// the hexahedron8 shape functions at point l (hexahedron.cpp:10-67, corner and point order as in
// make_hex8); inverted by Gauss-Jordan elimination with partial pivoting.  tet4 with one point:
// E = ones(4, 1) (tetrahedron.cpp:38-43).  E is [npe][nq].
static std::vector<double> extrapolation_matrix(int npe) {
    if (npe == 4) return {1.0, 1.0, 1.0, 1.0};
    const double lc[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                             {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    const double g = 1.0 / std::sqrt(3.0);
    double A[8][16];
    for (int l = 0; l < 8; ++l) {
        for (int a = 0; a < 8; ++a)
            A[l][a] = 0.125 * (1.0 + lc[a][0] * g * lc[l][0]) * (1.0 + lc[a][1] * g * lc[l][1]) *
                      (1.0 + lc[a][2] * g * lc[l][2]);
        for (int a = 0; a < 8; ++a) A[l][8 + a] = (l == a) ? 1.0 : 0.0;
    }
    for (int c = 0; c < 8; ++c) {
        int piv = c;
        for (int r = c + 1; r < 8; ++r)
            if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
        for (int k = 0; k < 16; ++k) std::swap(A[c][k], A[piv][k]);
        const double d = A[c][c];
        for (int k = 0; k < 16; ++k) A[c][k] /= d;
        for (int r = 0; r < 8; ++r) {
            if (r == c) continue;
            const double f = A[r][c];
            for (int k = 0; k < 16; ++k) A[r][k] -= f * A[c][k];
        }
    }
    std::vector<double> E(64);  // E[a][l] = (N^-1)[a][l]
    for (int a = 0; a < 8; ++a)
        for (int l = 0; l < 8; ++l) E[a * 8 + l] = A[a][8 + l];
    return E;
}

// submesh::nodal_averaged_variable (mesh/mechanics/solid/submesh.cpp:271-344) followed by
// average_internal_variable (io/post/node_averaged_variables.hpp:18-41): element by element the
// point values of each component are extrapolated with E and added to the element's nodes,
// each addition counted; the nodal value is the sum over the count.
// which: 0 Cauchy stress [N][9], 1 det F [N], 2 plastic strain [N][9],
//        3 accumulated plastic strain [N], 4 von Mises stress [N]
// unit-load vector of a non-follower load (kind 0 traction, 1 pressure, 2 body force); f [3N]
// is overwritten
void orc_nonfollower_load(void* h, int kind, int component, const int* faces, int nfaces, int npf,
                          int reduced, double* f) {
    const Oracle& o = *static_cast<Oracle*>(h);
    std::fill(f, f + o.ndofs(), 0.0);
    nonfollower_load(o, kind, component, faces, nfaces, npf, reduced, f);
}

int orc_nodal_average(void* h, int which, double* out) {
    auto* o = static_cast<Oracle*>(h);
    const std::vector<double>* v = nullptr;
    int nc = 1;
    switch (which) {
        case 0: v = &o->sigma; nc = 9; break;
        case 1: v = &o->detF; break;
        case 2: v = &o->ep; nc = 9; break;
        case 3: v = &o->epbar; break;
        case 4: v = &o->vm; break;
        default: return 1;
    }
    const std::vector<double> E = extrapolation_matrix(o->npe);
    std::vector<double> value((size_t)o->N * nc, 0.0), count((size_t)o->N * nc, 0.0);
    const int nq = o->nq, npe = o->npe;
    std::vector<double> comp(nq);
    for (int e = 0; e < o->E; ++e) {
        const int* nodes = &o->conn[(size_t)e * npe];
        for (int c = 0; c < nc; ++c) {
            for (int l = 0; l < nq; ++l) {
                const size_t q = (size_t)e * nq + l;
                comp[l] = v->empty() ? 0.0 : (*v)[q * nc + c];
            }
            for (int a = 0; a < npe; ++a) {
                double t = 0.0;
                for (int l = 0; l < nq; ++l) t += E[a * nq + l] * comp[l];
                value[(size_t)nodes[a] * nc + c] += t;
                count[(size_t)nodes[a] * nc + c] += 1.0;
            }
        }
    }
    for (size_t i = 0; i < value.size(); ++i) out[i] = value[i] / count[i];
    return 0;
}

}  // extern "C"
