// elements.cu -- fused element kernel for sm_100a: deformation measures, constitutive update at
// every quadrature point, tangent stiffness and internal force, scattered into the block CSR.
//
// Reference path (dbeurle/neon):
//   submesh::update_deformation_measures      src/mesh/mechanics/solid/submesh.cpp:210-237
//   submesh::update_Jacobian_determinants     submesh.cpp:239-269
//   constitutive updates                      src/constitutive/mechanics/solid/*.cpp (4 models)
//   submesh::material_tangent_stiffness       submesh.cpp:136-160   (sum_q B^T D B det J w)
//   submesh::geometric_tangent_stiffness      submesh.cpp:110-134   (sum_q L^T sigma L det J w, x I3)
//   submesh::internal_force                   submesh.cpp:82-108
//   static_matrix::assemble_stiffness         src/assembler/mechanics/static_matrix.hpp:243-277
//
// Work decomposition (hex8): a group of 8 lanes owns one element, 4 elements per warp.
//   phase 0  lane a gathers node a (X, u -> x = u + X) into shared memory;
//   phase 1  lane l runs quadrature point l in FP64: F0 = X dN, F = x dN, H, F F0^-1, det F check,
//            the constitutive update (J2 state read/written SoA, coalesced across lanes), the
//            current-configuration gradient L = dN J^-1 and the per-point tangent coefficients;
//   phase 2  lane g accumulates its 4-5 of the 36 upper-triangular 3x3 blocks over the 8 points.
//            All four models have an isotropic tangent in this formulation, plus a rank-one
//            deviatoric term for plastic J2, so a block is
//              K_ab = s[lam' La(x)Lb + mu'((La.Lb) I + Lb(x)La) + b (N La)(x)(N Lb)]
//                     + s (La.sigma.Lb) I   (finite strain)
//            which equals B_a^T D B_b det J w of the reference for
//              LE/J2 elastic  D = lam 1(x)1 + 2G I            (isotropic_linear_elasticity.cpp:55-67)
//              J2 plastic     D = C_e - c1 I_dev + c2 n(x)n   -> lam' = lam + c1/3, mu' = G - c1/2
//              neo-Hooke      D = lam 1(x)1 + 2(mu - lam ln J) I (compressible_neohooke.cpp:58-88)
//              microsphere    D = (k+p)1(x)1 - 2p I + P Dbar P with P(tau(x)1)P = 0 and
//                             P I P = I_dev -> lam' = k + p - 2/9 tr tau, mu' = tr tau/3 - p
//                             (gaussian_affine_microsphere.cpp:58-74);
//              Langevin       the same isotropic part plus the projected macro moduli
//              microsphere    P Cbar P = sum_i c_i m_i (x) m_i (m_i = dev(t_i (x) t_i)), a
//                             general symmetric 6x6 Da (affine_microsphere.cpp:58-112):
//                             K_ab += s B_a^T Da B_b;
//            the stiffness phase runs in Real (FP64 for parity, FP32 for the mixed path);
//   phase 3  each lane adds its blocks (and the mirrored lower blocks) with red.global.add into
//            K[slot], and the force of one node into f_int.
#include <cmath>
#include <utility>

#include "nb2_internal.cuh"

namespace nb2 {

__constant__ double c_dN_hex8[8 * 8 * 3];
__constant__ double c_w_hex8[8];
__constant__ double c_hex8_g;  // 1/sqrt(3) as the host computed it for c_dN_hex8
__constant__ double c_dN_tet4[4 * 3];
__constant__ float c_dNf_hex8[8 * 8 * 3];  // FP32 copies for the matrix-free FP32 operator
__constant__ float c_dNf_tet4[4 * 3];
// unit-sphere rules of the microsphere models, side by side: BO21 at 0, BO33 at 21
__constant__ double c_sphere_r[(21 + 33) * 3];
__constant__ double c_sphere_w[21 + 33];

// (row, first column, count) of the upper-triangular blocks owned by each lane of a group
__constant__ int c_seg_hex8[8][6] = {{0, 0, 5, 0, 0, 0}, {0, 5, 3, 7, 7, 1}, {1, 1, 5, 0, 0, 0},
                                     {1, 6, 2, 6, 6, 2}, {2, 2, 5, 0, 0, 0}, {2, 7, 1, 5, 5, 3},
                                     {3, 3, 5, 0, 0, 0}, {4, 4, 4, 0, 0, 0}};
__constant__ int c_seg_tet4[2][6] = {{0, 0, 4, 3, 3, 1}, {1, 1, 3, 2, 2, 2}};

template <int NPE>
struct Topo;
template <>
struct Topo<8> {
    static constexpr int NQ = 8, G = 8, EPC = 8, MAXB = 5;
};
template <>
struct Topo<4> {
    static constexpr int NQ = 1, G = 2, EPC = 32, MAXB = 5;
};

// ---------------------------------------------------------------------------------------
// 3x3 helpers (row-major).  Determinant: first-row expansion; inverse: cofactors times 1/det
// with det from the first column -- the fixed-size formulas of the reference's linear algebra.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double det3(const double* m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}

__device__ __forceinline__ void inv3(const double* m, double* r) {
    double c00 = m[4] * m[8] - m[5] * m[7];
    double c10 = m[7] * m[2] - m[8] * m[1];
    double c20 = m[1] * m[5] - m[2] * m[4];
    double det = c00 * m[0] + c10 * m[3] + c20 * m[6];
    double id = 1.0 / det;
    r[0] = c00 * id;
    r[1] = c10 * id;
    r[2] = c20 * id;
    r[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    r[4] = (m[8] * m[0] - m[6] * m[2]) * id;
    r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    r[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    r[7] = (m[6] * m[1] - m[7] * m[0]) * id;
    r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

// inverse as inv3, returning the determinant of m (the cofactor expansion along the first column)
__device__ __forceinline__ double inv3_det(const double* m, double* r) {
    double c00 = m[4] * m[8] - m[5] * m[7];
    double c10 = m[7] * m[2] - m[8] * m[1];
    double c20 = m[1] * m[5] - m[2] * m[4];
    double det = c00 * m[0] + c10 * m[3] + c20 * m[6];
    double id = 1.0 / det;
    r[0] = c00 * id;
    r[1] = c10 * id;
    r[2] = c20 * id;
    r[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    r[4] = (m[8] * m[0] - m[6] * m[2]) * id;
    r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    r[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    r[7] = (m[6] * m[1] - m[7] * m[0]) * id;
    r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
    return det;
}

__device__ __forceinline__ void matmul3(const double* a, const double* b, double* c) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            c[i * 3 + j] = a[i * 3 + 0] * b[0 * 3 + j] + a[i * 3 + 1] * b[1 * 3 + j] +
                           a[i * 3 + 2] * b[2 * 3 + j];
}

// symmetric tensor as 6 values (11, 22, 33, 23, 13, 12)
__device__ __forceinline__ double dev_norm6(const double* s) {
    double tr = (s[0] + s[1] + s[2]) / 3.0;
    double d0 = s[0] - tr, d1 = s[1] - tr, d2 = s[2] - tr;
    return sqrt(d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

struct QpOut {
    double sig[6];  // Cauchy stress
    double lam, mu, b;
    double N[6];    // J2 flow direction (plastic points)
    double Da[21];  // Langevin microsphere: anisotropic tangent, packed upper triangle (sym6)
};

// ----- constitutive models (FP64) --------------------------------------------------------

// isotropic_linear_elasticity.cpp:27-67
__device__ __forceinline__ void cm_linear_elastic(const ElementArgs& A, const double* H, QpOut& o) {
    double e0 = H[0], e1 = H[4], e2 = H[8];
    double e3 = 0.5 * (H[5] + H[7]), e4 = 0.5 * (H[2] + H[6]), e5 = 0.5 * (H[1] + H[3]);
    double tr = e0 + e1 + e2;
    o.sig[0] = A.lambda * tr + 2.0 * A.G * e0;
    o.sig[1] = A.lambda * tr + 2.0 * A.G * e1;
    o.sig[2] = A.lambda * tr + 2.0 * A.G * e2;
    o.sig[3] = 2.0 * A.G * e3;
    o.sig[4] = 2.0 * A.G * e4;
    o.sig[5] = 2.0 * A.G * e5;
    o.lam = A.lambda;
    o.mu = A.G;
    o.b = 0.0;
}

// compressible_neohooke.cpp:17-90
__device__ __forceinline__ void cm_neo_hooke(const ElementArgs& A, const double* F, double J,
                                             QpOut& o) {
    double B[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            B[i * 3 + j] = F[i * 3 + 0] * F[j * 3 + 0] + F[i * 3 + 1] * F[j * 3 + 1] +
                           F[i * 3 + 2] * F[j * 3 + 2];
    double lnJ = log(J);
    double mu = A.G, lam = A.lambda;
    o.sig[0] = (lam * lnJ + mu * (B[0] - 1.0)) / J;
    o.sig[1] = (lam * lnJ + mu * (B[4] - 1.0)) / J;
    o.sig[2] = (lam * lnJ + mu * (B[8] - 1.0)) / J;
    o.sig[3] = (mu * B[5]) / J;
    o.sig[4] = (mu * B[2]) / J;
    o.sig[5] = (mu * B[1]) / J;
    o.lam = lam;
    o.mu = mu - lam * lnJ;
    o.b = 0.0;
}

// small_strain_J2_plasticity.cpp:30-163; the current plastic state is mutated on every call.
// ep_in / ebar_in: the point's plastic strain and accumulated plastic strain, loaded by the
// caller ahead of its geometry so the loads overlap it
__device__ __forceinline__ bool cm_j2(const ElementArgs& A, long long q, const double* H,
                                      QpOut& o, const double* ep_in, double ebar_in) {
    const double G = A.G, lam = A.lambda, Hh = A.H_iso;
    const long long n = A.nqp;
    double ep[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) ep[c] = ep_in[c];
    double ebar = ebar_in;
    double e0 = H[0] - ep[0], e1 = H[4] - ep[1], e2 = H[8] - ep[2];
    double e3 = 0.5 * (H[5] + H[7]) - ep[3], e4 = 0.5 * (H[2] + H[6]) - ep[4],
           e5 = 0.5 * (H[1] + H[3]) - ep[5];
    double tr = e0 + e1 + e2;
    double* s = o.sig;
    s[0] = lam * tr + 2.0 * G * e0;
    s[1] = lam * tr + 2.0 * G * e1;
    s[2] = lam * tr + 2.0 * G * e2;
    s[3] = 2.0 * G * e3;
    s[4] = 2.0 * G * e4;
    s[5] = 2.0 * G * e5;
    const double dn = dev_norm6(s);
    const double vm = sqrt(3.0 / 2.0) * dn;
    o.lam = lam;
    o.mu = G;
    o.b = 0.0;
    double f = (vm - 3.0 * G * 0.0) - (A.sigma_y + ebar * Hh);
    if (f <= 0.0) return true;
    const double vm_trial = vm;
    double trs = (s[0] + s[1] + s[2]) / 3.0;
    double nrm[6] = {(s[0] - trs) / dn, (s[1] - trs) / dn, (s[2] - trs) / dn,
                     s[3] / dn,         s[4] / dn,         s[5] / dn};
    double dg = 0.0;
    int it = 0;
    while (f > 1.0e-6 && it < 50) {
        dg += f / (3.0 * G + Hh);
        f = (vm - 3.0 * G * dg) - (A.sigma_y + (ebar + dg) * Hh);
        ++it;
    }
    if (it == 50) return false;
    const double s32 = sqrt(3.0 / 2.0);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        A.ep[c * n + q] = ep[c] + dg * s32 * nrm[c];
        s[c] -= 2.0 * G * dg * s32 * nrm[c];
    }
    A.epbar[q] = ebar + dg;
    double c1 = dg * 6.0 * (G * G) / vm_trial;
    double c2 = 6.0 * (G * G) * (dg / vm_trial - 1.0 / (3.0 * G + Hh));
    o.lam = lam + c1 / 3.0;
    o.mu = G - 0.5 * c1;
    o.b = c2;
#pragma unroll
    for (int c = 0; c < 6; ++c) o.N[c] = nrm[c];
    return true;
}

// gaussian_affine_microsphere.cpp:23-88 with volumetric_free_energy.hpp:16-30
__device__ __forceinline__ void cm_microsphere(const ElementArgs& A, double Gm, const double* F,
                                               double J, QpOut& o) {
    const double K = A.K;
    double sc = pow(det3(F), -1.0 / 3.0);
    double Fb[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Fb[i] = sc * F[i];
    double acc[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 3
    for (int i = A.sph0; i < A.sph0 + A.nsph; ++i) {
        double r0 = c_sphere_r[3 * i], r1 = c_sphere_r[3 * i + 1], r2 = c_sphere_r[3 * i + 2];
        double w = c_sphere_w[i];
        double t0 = Fb[0] * r0 + Fb[1] * r1 + Fb[2] * r2;
        double t1 = Fb[3] * r0 + Fb[4] * r1 + Fb[5] * r2;
        double t2 = Fb[6] * r0 + Fb[7] * r1 + Fb[8] * r2;
        acc[0] += (t0 * t0) * w;
        acc[1] += (t1 * t1) * w;
        acc[2] += (t2 * t2) * w;
        acc[3] += (t1 * t2) * w;
        acc[4] += (t0 * t2) * w;
        acc[5] += (t0 * t1) * w;
    }
    double tau[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) tau[c] = 3.0 * Gm * acc[c];
    double p = J * (K / 2.0 * (J - 1.0 / J));
    double trt = tau[0] + tau[1] + tau[2];
    double tr3 = trt / 3.0;
    o.sig[0] = (p + tau[0] - tr3) / J;
    o.sig[1] = (p + tau[1] - tr3) / J;
    o.sig[2] = (p + tau[2] - tr3) / J;
    o.sig[3] = tau[3] / J;
    o.sig[4] = tau[4] / J;
    o.sig[5] = tau[5] / J;
    double kappa = (J * J) * (K / 2.0 * (1.0 + 1.0 / (J * J)));
    o.lam = kappa + p - (2.0 / 9.0) * trt;
    o.mu = trt / 3.0 - p;
    o.b = 0.0;
}

// affine_microsphere.cpp:23-112 with the Pade approximants of detail/microsphere.hpp:40-70.
// Per sphere direction r_i: t = Fbar r_i, l^2 = t.t, d = N - l^2,
//   pade_first  = (3N - l^2) / d,   pade_second = (l^4 + 3N^2) / d^2,
//   tau    = G sum_i w_i pade_first t (x) t,
//   Cbar   = G sum_i w_i l^-2 (pade_second - pade_first) t(x)t(x)t(x)t.
// The tangent (k + p) 1(x)1 - 2p I + P (Cbar + 2/3 tr tau I - 2/3 (tau(x)1 + 1(x)tau)) P splits
// as for the Gaussian model into lam', mu' and the projected macro moduli
//   Da = P Cbar P = G sum_i w_i l^-2 (pade_second - pade_first) m_i (x) m_i,  m_i = dev(t (x) t)
// (P t(x)t = dev(t(x)t) in kinetic Voigt), accumulated directly as a packed 6x6.
__device__ __forceinline__ void cm_langevin(const ElementArgs& A, double Gm, const double* F,
                                            double J, QpOut& o) {
    const double K = A.K, Nc = A.Nseg;
    double sc = pow(det3(F), -1.0 / 3.0);
    double Fb[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Fb[i] = sc * F[i];
    double acc[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int c = 0; c < 21; ++c) o.Da[c] = 0.0;
#pragma unroll 1
    for (int i = A.sph0; i < A.sph0 + A.nsph; ++i) {
        double r0 = c_sphere_r[3 * i], r1 = c_sphere_r[3 * i + 1], r2 = c_sphere_r[3 * i + 2];
        double w = c_sphere_w[i];
        double t0 = Fb[0] * r0 + Fb[1] * r1 + Fb[2] * r2;
        double t1 = Fb[3] * r0 + Fb[4] * r1 + Fb[5] * r2;
        double t2 = Fb[6] * r0 + Fb[7] * r1 + Fb[8] * r2;
        const double l2 = t0 * t0 + t1 * t1 + t2 * t2;
        const double d = Nc - l2;
        const double pf = (3.0 * Nc - l2) / d;
        const double ps = (l2 * l2 + 3.0 * Nc * Nc) / (d * d);
        const double wf = w * pf;
        acc[0] += (t0 * t0) * wf;
        acc[1] += (t1 * t1) * wf;
        acc[2] += (t2 * t2) * wf;
        acc[3] += (t1 * t2) * wf;
        acc[4] += (t0 * t2) * wf;
        acc[5] += (t0 * t1) * wf;
        const double a4 = Gm * w * (ps - pf) / l2;
        const double l3 = l2 / 3.0;
        const double m[6] = {t0 * t0 - l3, t1 * t1 - l3, t2 * t2 - l3, t1 * t2, t0 * t2, t0 * t1};
#pragma unroll
        for (int v = 0; v < 6; ++v)
#pragma unroll
            for (int u = v; u < 6; ++u) o.Da[sym6(v, u)] += a4 * m[v] * m[u];
    }
    double tau[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) tau[c] = Gm * acc[c];
    double p = J * (K / 2.0 * (J - 1.0 / J));
    double trt = tau[0] + tau[1] + tau[2];
    double tr3 = trt / 3.0;
    o.sig[0] = (p + tau[0] - tr3) / J;
    o.sig[1] = (p + tau[1] - tr3) / J;
    o.sig[2] = (p + tau[2] - tr3) / J;
    o.sig[3] = tau[3] / J;
    o.sig[4] = tau[4] / J;
    o.sig[5] = tau[5] / J;
    double kappa = (J * J) * (K / 2.0 * (1.0 + 1.0 / (J * J)));
    o.lam = kappa + p - (2.0 / 9.0) * trt;
    o.mu = trt / 3.0 - p;
    o.b = 0.0;
}

// P C P for a packed symmetric 6x6 C in kinetic Voigt, P the deviatoric projector (normal block
// I - 1/3 1 1^T, shear block I): subtract the normal-row means on both sides
__device__ __forceinline__ void project_deviatoric(const double* C, double* Da) {
    double cm[6];
#pragma unroll
    for (int w = 0; w < 6; ++w) cm[w] = (C[sym6(0, w)] + C[sym6(1, w)] + C[sym6(2, w)]) / 3.0;
    const double mm = (cm[0] + cm[1] + cm[2]) / 3.0;
#pragma unroll
    for (int v = 0; v < 6; ++v)
#pragma unroll
        for (int w = v; w < 6; ++w) {
            double d = C[sym6(v, w)];
            if (v < 3 && w < 3)
                d += mm - cm[v] - cm[w];
            else if (v < 3)
                d -= cm[w];
            Da[sym6(v, w)] = d;
        }
}

// nonaffine_microsphere.cpp:29-175 (tube geometry U = 9 and tube parameter q = 1 are members of
// the reference class; the stretch parameter p comes from the material).  One pass over the 21
// directions accumulates, with t = Fbar r, l = |t|, n = Fbar^-T r, nu = |n|:
//   sum w l^p,  h = sum w l^(p-2) t(x)t,  H/(p-2) = sum w l^(p-4) t(x)t(x)t(x)t,
//   k = sum w nu^-1 n(x)n,  K + G = sum w (-nu^-3 n(x)n(x)n(x)n + 2 nu^-1 o(n))   (q = 1);
// then lambda = (sum w l^p)^(1/p) and, with pf, ps the Pade approximants at lambda,
//   tau = G pf lambda^(2-p) h - G N U k,
//   C   = (G ps - (p-1) G pf) lambda^(2-2p) h(x)h + G pf lambda^(2-p) H + G N U (K + G);
// the tangent is the affine model's: lam', mu' from tau and Da = P C P.
__device__ __forceinline__ void cm_nonaffine(const ElementArgs& A, double Gm, const double* F,
                                             double J, QpOut& o) {
    constexpr double U = 9.0;
    const double K = A.K, Nc = A.Nseg, pp = A.p_na;
    const double sc = pow(det3(F), -1.0 / 3.0);
    double Fb[9], Fbi[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Fb[i] = sc * F[i];
    inv3(Fb, Fbi);
    double lp = 0.0, h[6] = {0, 0, 0, 0, 0, 0}, k[6] = {0, 0, 0, 0, 0, 0};
    double H[21], C[21];
#pragma unroll
    for (int c = 0; c < 21; ++c) H[c] = C[c] = 0.0;
#pragma unroll 1
    for (int i = A.sph0; i < A.sph0 + A.nsph; ++i) {
        const double r0 = c_sphere_r[3 * i], r1 = c_sphere_r[3 * i + 1], r2 = c_sphere_r[3 * i + 2];
        const double w = c_sphere_w[i];
        const double t[3] = {Fb[0] * r0 + Fb[1] * r1 + Fb[2] * r2,
                             Fb[3] * r0 + Fb[4] * r1 + Fb[5] * r2,
                             Fb[6] * r0 + Fb[7] * r1 + Fb[8] * r2};
        const double n[3] = {Fbi[0] * r0 + Fbi[3] * r1 + Fbi[6] * r2,
                             Fbi[1] * r0 + Fbi[4] * r1 + Fbi[7] * r2,
                             Fbi[2] * r0 + Fbi[5] * r1 + Fbi[8] * r2};
        const double l2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
        const double nu = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        const double lpw = pow(sqrt(l2), pp);
        lp += lpw * w;
        const double a2 = w * lpw / l2, a4 = a2 / l2;      // w l^(p-2), w l^(p-4)
        const double b1 = w / nu, b3 = b1 / (nu * nu);      // w nu^-1, w nu^-3
        const double tv[6] = {t[0] * t[0], t[1] * t[1], t[2] * t[2], t[1] * t[2], t[0] * t[2],
                              t[0] * t[1]};
        const double nv[6] = {n[0] * n[0], n[1] * n[1], n[2] * n[2], n[1] * n[2], n[0] * n[2],
                              n[0] * n[1]};
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            h[c] += a2 * tv[c];
            k[c] += b1 * nv[c];
        }
#pragma unroll
        for (int v = 0; v < 6; ++v)
#pragma unroll
            for (int u = v; u < 6; ++u) {
                H[sym6(v, u)] += a4 * tv[v] * tv[u];
                C[sym6(v, u)] -= b3 * nv[v] * nv[u];
            }
        // 2 o(n) (compute_o_dot_product), upper triangle
        const double b2 = 2.0 * b1;
        C[sym6(0, 0)] += b2 * 2.0 * nv[0];
        C[sym6(1, 1)] += b2 * 2.0 * nv[1];
        C[sym6(2, 2)] += b2 * 2.0 * nv[2];
        C[sym6(0, 4)] += b2 * nv[4];
        C[sym6(0, 5)] += b2 * nv[5];
        C[sym6(1, 3)] += b2 * nv[3];
        C[sym6(1, 5)] += b2 * nv[5];
        C[sym6(2, 3)] += b2 * nv[3];
        C[sym6(2, 4)] += b2 * nv[4];
        C[sym6(3, 3)] += b2 * 0.5 * (nv[1] + nv[2]);
        C[sym6(3, 4)] += b2 * 0.5 * nv[5];
        C[sym6(3, 5)] += b2 * 0.5 * nv[4];
        C[sym6(4, 4)] += b2 * 0.5 * (nv[0] + nv[2]);
        C[sym6(4, 5)] += b2 * 0.5 * nv[3];
        C[sym6(5, 5)] += b2 * 0.5 * (nv[0] + nv[1]);
    }
    const double lam = pow(lp, 1.0 / pp);
    const double d = Nc - lam * lam;
    const double pf = (3.0 * Nc - lam * lam) / d;
    const double ps = (lam * lam * lam * lam + 3.0 * Nc * Nc) / (d * d);
    const double micro_tau = Gm * pf * lam;
    const double cf = micro_tau * pow(lam, 1.0 - pp);
    const double chh = Gm * ps * pow(lam, 2.0 - 2.0 * pp) -
                       (pp - 1.0) * micro_tau * pow(lam, 1.0 - 2.0 * pp);
    const double gnu = Gm * Nc * U;
    double tau[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) tau[c] = cf * h[c] - gnu * k[c];
#pragma unroll
    for (int v = 0; v < 6; ++v)
#pragma unroll
        for (int u = v; u < 6; ++u)
            C[sym6(v, u)] = chh * h[v] * h[u] + cf * (pp - 2.0) * H[sym6(v, u)] + gnu * C[sym6(v, u)];
    project_deviatoric(C, o.Da);
    const double p = J * (K / 2.0 * (J - 1.0 / J));
    const double trt = tau[0] + tau[1] + tau[2];
    const double tr3 = trt / 3.0;
    o.sig[0] = (p + tau[0] - tr3) / J;
    o.sig[1] = (p + tau[1] - tr3) / J;
    o.sig[2] = (p + tau[2] - tr3) / J;
    o.sig[3] = tau[3] / J;
    o.sig[4] = tau[4] / J;
    o.sig[5] = tau[5] / J;
    const double kappa = (J * J) * (K / 2.0 * (1.0 + 1.0 / (J * J)));
    o.lam = kappa + p - (2.0 / 9.0) * trt;
    o.mu = trt / 3.0 - p;
    o.b = 0.0;
}

// y += B_a^T Da B_b restricted to one 3x3 block: K[i][k] += sum_vw B_a[v][i] Da[v][w] B_b[w][k]
// with the kinematic strain operator B (rows 11 22 33 23 13 12; shear rows engineering).
// Column k of B_b has three entries: k=0 -> rows (0, 4, 5) = (L0, L2, L1), k=1 -> (1, 3, 5) =
// (L1, L2, L0), k=2 -> (2, 3, 4) = (L2, L1, L0).
template <typename Real, typename DaT>
__device__ __forceinline__ void aniso_block(const DaT* Da, const Real* La, const Real* Lb,
                                            Real* acc) {
    Real Z[6][3];
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        Z[v][0] = (Real)Da[sym6(v, 0)] * Lb[0] + (Real)Da[sym6(v, 4)] * Lb[2] +
                  (Real)Da[sym6(v, 5)] * Lb[1];
        Z[v][1] = (Real)Da[sym6(v, 1)] * Lb[1] + (Real)Da[sym6(v, 3)] * Lb[2] +
                  (Real)Da[sym6(v, 5)] * Lb[0];
        Z[v][2] = (Real)Da[sym6(v, 2)] * Lb[2] + (Real)Da[sym6(v, 3)] * Lb[1] +
                  (Real)Da[sym6(v, 4)] * Lb[0];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        acc[0 * 3 + k] += La[0] * Z[0][k] + La[2] * Z[4][k] + La[1] * Z[5][k];
        acc[1 * 3 + k] += La[1] * Z[1][k] + La[2] * Z[3][k] + La[0] * Z[5][k];
        acc[2 * 3 + k] += La[2] * Z[2][k] + La[1] * Z[3][k] + La[0] * Z[4][k];
    }
}

// sigma_a = Da eps with eps the engineering strain of the gradient G (row-major 3x3); returns
// the symmetric stress in kinetic Voigt order
template <typename Real, typename DaT>
__device__ __forceinline__ void aniso_stress(const DaT* Da, const Real* G, Real* sa) {
    const Real eps[6] = {G[0], G[4], G[8], G[5] + G[7], G[2] + G[6], G[1] + G[3]};
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        Real t = (Real)0;
#pragma unroll
        for (int w = 0; w < 6; ++w) t += (Real)Da[sym6(v, w)] * eps[w];
        sa[v] = t;
    }
}

// The material moduli of element e: per-element shear / bulk modulus when given (batched
// instances of different materials, per-element parameter fields), else the material's.
__device__ __forceinline__ ElementArgs element_moduli(const ElementArgs& A, long long e) {
    ElementArgs Ae = A;
    if (A.Ge || A.Ke) {
        if (A.Ge) Ae.G = A.Ge[e];
        if (A.Ke) Ae.K = A.Ke[e];
        Ae.lambda = Ae.K - 2.0 * Ae.G / 3.0;
    }
    return Ae;
}

__device__ __forceinline__ void report_status(const ElementArgs& A, long long e, int code) {
    atomicOr(&A.status->flags, 1u << (code - 1));
    if (A.inst_flags) atomicOr(&A.inst_flags[A.e_inst[e]], 1u << (code - 1));
}

// batched solves compute only the elements of the instances still iterating
__device__ __forceinline__ bool element_enabled(const ElementArgs& A, long long e) {
    return e >= 0 && e < A.E && (A.inst_on == nullptr || A.inst_on[A.e_inst[e]] != 0);
}

// the element at position pos of this launch: the pos-th element of the launch's colour in a
// colour-partitioned pass, else element pos; -1 past the end
__device__ __forceinline__ long long element_at(const ElementArgs& A, long long pos) {
    if (pos >= A.ecount) return -1;
    return A.order ? (long long)A.order[pos] : pos;
}

// D += A B for one 8x8x4 FP64 tile (mma.sync m8n8k4, row.col): lane l holds A[l/4][l%4],
// B[l%4][l/4] and D[l/4][2(l%4) + {0, 1}]
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// hexahedron8 shape-function derivatives at one point of the 8-point rule, in registers: the
// point's factors 1 + s x (s = -1, +1 for each reference coordinate x) are formed once, and each
// derivative is the product the host table c_dN_hex8 evaluates, in its order, so the values are
// the same bits (hexahedron.cpp:10-67).  The fused element kernel uses it instead of a shared
// table, whose broadcast reads cost two shared-memory wavefronts per 64-bit load.
struct Hex8Point {
    double f[3][2];  // [reference coordinate][s = -1, +1]
};

__device__ __forceinline__ Hex8Point hex8_point(int l) {
    const double g = c_hex8_g;
    const double x = ((l == 1) || (l == 2) || (l == 5) || (l == 6)) ? g : -g;
    const double e = ((l == 2) || (l == 3) || (l == 6) || (l == 7)) ? g : -g;
    const double z = (l >= 4) ? g : -g;
    Hex8Point P;
    P.f[0][0] = 1.0 + (-1.0) * x;
    P.f[0][1] = 1.0 + 1.0 * x;
    P.f[1][0] = 1.0 + (-1.0) * e;
    P.f[1][1] = 1.0 + 1.0 * e;
    P.f[2][0] = 1.0 + (-1.0) * z;
    P.f[2][1] = 1.0 + 1.0 * z;
    return P;
}

// dN_a / dxi_k (a, k known at compile time once the callers' loops unroll)
__device__ __forceinline__ double hex8_dN(const Hex8Point& P, int a, int k) {
    const int sx = ((a == 1) || (a == 2) || (a == 5) || (a == 6)) ? 1 : 0;
    const int se = ((a == 2) || (a == 3) || (a == 6) || (a == 7)) ? 1 : 0;
    const int sz = (a >= 4) ? 1 : 0;
    const double xa = sx ? 1.0 : -1.0, ea = se ? 1.0 : -1.0, za = sz ? 1.0 : -1.0;
    if (k == 0) return 1.0 / 8.0 * xa * P.f[1][se] * P.f[2][sz];
    if (k == 1) return 1.0 / 8.0 * P.f[0][sx] * ea * P.f[2][sz];
    return 1.0 / 8.0 * P.f[0][sx] * P.f[1][se] * za;
}

#include "element_kernel.cuh"

// ---------------------------------------------------------------------------------------
// Matrix-free FP64 product y += K v with the tangent of the last stored update: the defect
// residual of the mixed-precision solve.  With G = sum_b v_b (x) L_b (the gradient of v) the
// element force of node a is
//   y_a = s [lam' tr(G) La + mu' (G + G^T) La + b (N:G) N La + (Da eps(G)) La + G sigma La]
// -- the same tangent the assembled K holds, applied without forming it.
// ---------------------------------------------------------------------------------------
// The stored tangent applied at one quadrature point: for the gradient Gm = sum_a v_a (x) L_a of
// an input v, out[3a + i] = s t_a[i] with
//   t_a = lam' tr(G) La + mu' (G + G^T) La + b (N:G) N La + (Da eps(G)) La + G sigma La,
// the point's share of (K_e v)_a (the block formula of the assembled tangent, applied)
template <int NPE, int MODEL>
__device__ __forceinline__ void tangent_point_product(const ElementArgs& A, long long q, double s,
                                                      const double (&L)[NPE][3], const double* Gm,
                                                      double* out) {
    constexpr bool kFinite = (MODEL == MODEL_NH || MODEL == MODEL_MS || model_aniso(MODEL));
    constexpr bool kJ2 = (MODEL == MODEL_J2);
    constexpr bool kAniso = model_aniso(MODEL);
    const long long n = A.nqp;
    const double lam = A.dpar[0 * n + q], mu = A.dpar[1 * n + q];
    const double trG = Gm[0] + Gm[4] + Gm[8];
    double bN = 0.0, N6[6] = {0, 0, 0, 0, 0, 0};
    if constexpr (kJ2) {
        const double b = A.dpar[2 * n + q];
        if (b != 0.0) {
#pragma unroll
            for (int c = 0; c < 6; ++c) N6[c] = A.dpar[(3 + c) * n + q];
            // N:G with N symmetric (11 22 33 23 13 12)
            bN = b * (N6[0] * Gm[0] + N6[1] * Gm[4] + N6[2] * Gm[8] +
                      N6[3] * (Gm[5] + Gm[7]) + N6[4] * (Gm[2] + Gm[6]) +
                      N6[5] * (Gm[1] + Gm[3]));
        }
    }
    double sa[6] = {0, 0, 0, 0, 0, 0};
    if constexpr (kAniso) {
        double Da[21];
#pragma unroll
        for (int c = 0; c < 21; ++c) Da[c] = A.dpar[(3 + c) * n + q];
        aniso_stress(Da, Gm, sa);
    }
    double sg[6] = {0, 0, 0, 0, 0, 0};
    if constexpr (kFinite) {
#pragma unroll
        for (int c = 0; c < 6; ++c) sg[c] = A.sig[c * n + q];
    }
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
        const double* La = L[a];
        double t[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
            t[i] = lam * trG * La[i] +
                   mu * ((Gm[i * 3 + 0] + Gm[0 * 3 + i]) * La[0] +
                         (Gm[i * 3 + 1] + Gm[1 * 3 + i]) * La[1] +
                         (Gm[i * 3 + 2] + Gm[2 * 3 + i]) * La[2]);
        if constexpr (kJ2) {
            t[0] += bN * (N6[0] * La[0] + N6[5] * La[1] + N6[4] * La[2]);
            t[1] += bN * (N6[5] * La[0] + N6[1] * La[1] + N6[3] * La[2]);
            t[2] += bN * (N6[4] * La[0] + N6[3] * La[1] + N6[2] * La[2]);
        }
        if constexpr (kAniso) {
            t[0] += sa[0] * La[0] + sa[5] * La[1] + sa[4] * La[2];
            t[1] += sa[5] * La[0] + sa[1] * La[1] + sa[3] * La[2];
            t[2] += sa[4] * La[0] + sa[3] * La[1] + sa[2] * La[2];
        }
        if constexpr (kFinite) {
            const double sl0 = sg[0] * La[0] + sg[5] * La[1] + sg[4] * La[2];
            const double sl1 = sg[5] * La[0] + sg[1] * La[1] + sg[3] * La[2];
            const double sl2 = sg[4] * La[0] + sg[3] * La[1] + sg[2] * La[2];
#pragma unroll
            for (int i = 0; i < 3; ++i)
                t[i] += Gm[i * 3 + 0] * sl0 + Gm[i * 3 + 1] * sl1 + Gm[i * 3 + 2] * sl2;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) out[3 * a + i] = s * t[i];
    }
}

template <int NPE, int MODEL>
__global__ void __launch_bounds__(64) k_apply(ElementArgs A, const double* __restrict__ v,
                                              double* __restrict__ y) {
    using T = Topo<NPE>;
    constexpr int NQ = T::NQ, G = T::G, EPC = T::EPC;
    __shared__ double sx[EPC][NPE][3];
    __shared__ double sv[EPC][NPE][3];
    __shared__ double sdN[NQ][NPE][3];
    __shared__ double sY[EPC][NQ][NPE * 3];
    const int tid = threadIdx.x;
    const int le = tid / G;
    const int lane = tid % G;
    const long long e = element_at(A, (long long)blockIdx.x * EPC + le);
    const bool valid = element_enabled(A, e);
    for (int i = tid; i < NQ * NPE * 3; i += blockDim.x)
        (&sdN[0][0][0])[i] = (NPE == 8) ? c_dN_hex8[i] : c_dN_tet4[i];
    int node[(NPE + G - 1) / G];
#pragma unroll
    for (int j = 0; j < (NPE + G - 1) / G; ++j) {
        int a = lane + j * G;
        node[j] = 0;
        if (a < NPE && valid) {
            int nd = A.conn[e * NPE + a];
            node[j] = nd;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sx[le][a][k] = A.u[3ll * nd + k] + A.X[3ll * nd + k];
                sv[le][a][k] = v[3ll * nd + k];
            }
        }
    }
    __syncthreads();
    for (int l = lane; l < NQ; l += G) {
        if (!valid) break;
        const double w = (NPE == 8) ? c_w_hex8[l] : (1.0 / 6.0);
        const long long q = e * NQ + l;
        double Fc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) Fc[i * 3 + k] += sx[le][a][i] * sdN[l][a][k];
        double Ji[9];
        inv3(Fc, Ji);
        const double s = w * det3(Fc);
        double L[NPE][3];
        double Gm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 0; a < NPE; ++a) {
#pragma unroll
            for (int k = 0; k < 3; ++k)
                L[a][k] = sdN[l][a][0] * Ji[0 * 3 + k] + sdN[l][a][1] * Ji[1 * 3 + k] +
                          sdN[l][a][2] * Ji[2 * 3 + k];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) Gm[i * 3 + k] += sv[le][a][i] * L[a][k];
        }
        tangent_point_product<NPE, MODEL>(A, q, s, L, Gm, &sY[le][l][0]);
    }
    __syncthreads();
    if (!valid) return;
#pragma unroll
    for (int j = 0; j < (NPE + G - 1) / G; ++j) {
        int a = lane + j * G;
        if (a < NPE) {
            double f0 = 0, f1 = 0, f2 = 0;
#pragma unroll
            for (int l = 0; l < NQ; ++l) {
                f0 += sY[le][l][3 * a + 0];
                f1 += sY[le][l][3 * a + 1];
                f2 += sY[le][l][3 * a + 2];
            }
            atomicAdd(&y[3ll * node[j] + 0], f0);
            atomicAdd(&y[3ll * node[j] + 1], f1);
            atomicAdd(&y[3ll * node[j] + 2], f2);
        }
    }
}

// One element's tangent stiffness from the stored tangent of the last update, dense
// [3 NPE][3 NPE] row-major in neon's local DOF order (3a + k): thread j forms column j, the
// element product with the unit vector e_j, point by point (submesh::tangent_stiffness,
// submesh.cpp:66-80; a debug getter, one block)
template <int NPE, int MODEL>
__global__ void k_element_stiffness(ElementArgs A, long long e, double* __restrict__ Ke) {
    constexpr int NQ = Topo<NPE>::NQ, ND = 3 * NPE;
    const int j = threadIdx.x;
    if (j >= ND) return;
    double xa[NPE][3];
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
        const long long nd = A.conn[e * NPE + a];
#pragma unroll
        for (int k = 0; k < 3; ++k) xa[a][k] = A.u[3 * nd + k] + A.X[3 * nd + k];
    }
    double col[ND];
#pragma unroll
    for (int r = 0; r < ND; ++r) col[r] = 0.0;
    for (int l = 0; l < NQ; ++l) {
        const double* dN = (NPE == 8) ? &c_dN_hex8[l * 24] : c_dN_tet4;
        double Fc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) Fc[i * 3 + k] += xa[a][i] * dN[a * 3 + k];
        double Ji[9];
        inv3(Fc, Ji);
        const double s = ((NPE == 8) ? c_w_hex8[l] : (1.0 / 6.0)) * det3(Fc);
        double L[NPE][3];
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int k = 0; k < 3; ++k)
                L[a][k] = dN[a * 3 + 0] * Ji[0 * 3 + k] + dN[a * 3 + 1] * Ji[1 * 3 + k] +
                          dN[a * 3 + 2] * Ji[2 * 3 + k];
        // v = e_j: G = e_i (x) L_b with b = j / 3, i = j % 3
        double Gm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const int b = j / 3, i = j % 3;
#pragma unroll
        for (int k = 0; k < 3; ++k) Gm[i * 3 + k] = L[b][k];
        double out[ND];
        tangent_point_product<NPE, MODEL>(A, e * NQ + l, s, L, Gm, out);
#pragma unroll
        for (int r = 0; r < ND; ++r) col[r] += out[r];
    }
#pragma unroll
    for (int r = 0; r < ND; ++r) Ke[r * ND + j] = col[r];
}

#include "mf_kernels.cuh"

// ---------------------------------------------------------------------------------------
// Adjoint gradient with respect to the per-element shear modulus of the Gaussian or Langevin
// affine microsphere.  With K lambda = dJ/du solved on the converged tangent,
//   dJ/dG_e = - lambda^T df_int/dG_e = - sum_q s_q (d sigma_q / dG) : grad(lambda)_q,
// where sigma = (p I + dev tau)/J and tau = G sum_i w_i f_i t_i (x) t_i (t_i = Fbar r_i; chain
// weight f_i = 3 Gaussian, pade_first(|t_i|, N) Langevin), so
// d sigma/dG = dev(sum_i w_i f_i t_i (x) t_i) / J.  The quadrature-point state (F, Fbar, the
// sphere sum) is recomputed from the displacement, not stored.  One value per element: the
// group reduces over its points with shuffles, no atomics.
// ---------------------------------------------------------------------------------------
template <int NPE, int MODEL>
__global__ void __launch_bounds__(64) k_adjoint_shear(ElementArgs A, const double* __restrict__ lam,
                                                      double* __restrict__ dJdG) {
    using T = Topo<NPE>;
    constexpr int NQ = T::NQ, G = T::G, EPC = T::EPC;
    __shared__ double sX[EPC][NPE][3];
    __shared__ double sx[EPC][NPE][3];
    __shared__ double sl[EPC][NPE][3];
    __shared__ double sdN[NQ][NPE][3];
    const int tid = threadIdx.x;
    const int le = tid / G;
    const int lane = tid % G;
    const long long e = (long long)blockIdx.x * EPC + le;
    const bool valid = e < A.E;
    for (int i = tid; i < NQ * NPE * 3; i += blockDim.x)
        (&sdN[0][0][0])[i] = (NPE == 8) ? c_dN_hex8[i] : c_dN_tet4[i];
#pragma unroll
    for (int j = 0; j < (NPE + G - 1) / G; ++j) {
        const int a = lane + j * G;
        if (a < NPE && valid) {
            const int nd = A.conn[e * NPE + a];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double Xv = A.X[3ll * nd + k];
                sX[le][a][k] = Xv;
                sx[le][a][k] = A.u[3ll * nd + k] + Xv;
                sl[le][a][k] = lam[3ll * nd + k];
            }
        }
    }
    __syncthreads();
    double contrib = 0.0;
    const int l = lane;
    if (valid && l < NQ) {
        const double w = (NPE == 8) ? c_w_hex8[l] : (1.0 / 6.0);
        double Fc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, F0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    Fc[i * 3 + k] += sx[le][a][i] * sdN[l][a][k];
                    F0[i * 3 + k] += sX[le][a][i] * sdN[l][a][k];
                }
        double F0i[9], Fd[9], Ji[9];
        inv3(F0, F0i);
        matmul3(Fc, F0i, Fd);
        const double J = det3(Fd);
        const double sc = pow(J, -1.0 / 3.0);
        double acc[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 3
        for (int i = A.sph0; i < A.sph0 + A.nsph; ++i) {
            const double r0 = c_sphere_r[3 * i], r1 = c_sphere_r[3 * i + 1],
                         r2 = c_sphere_r[3 * i + 2], wi = c_sphere_w[i];
            const double t0 = sc * (Fd[0] * r0 + Fd[1] * r1 + Fd[2] * r2);
            const double t1 = sc * (Fd[3] * r0 + Fd[4] * r1 + Fd[5] * r2);
            const double t2 = sc * (Fd[6] * r0 + Fd[7] * r1 + Fd[8] * r2);
            double f = 3.0;
            if constexpr (MODEL == MODEL_ML) {
                const double l2 = t0 * t0 + t1 * t1 + t2 * t2;
                f = (3.0 * A.Nseg - l2) / (A.Nseg - l2);
            }
            const double wf = wi * f;
            acc[0] += (t0 * t0) * wf;
            acc[1] += (t1 * t1) * wf;
            acc[2] += (t2 * t2) * wf;
            acc[3] += (t1 * t2) * wf;
            acc[4] += (t0 * t2) * wf;
            acc[5] += (t0 * t1) * wf;
        }
        // d sigma / dG = dev(acc) / J  (11 22 33 23 13 12)
        const double tr3 = (acc[0] + acc[1] + acc[2]) / 3.0;
        double ds[6] = {(acc[0] - tr3) / J, (acc[1] - tr3) / J, (acc[2] - tr3) / J,
                        acc[3] / J,         acc[4] / J,         acc[5] / J};
        inv3(Fc, Ji);
        const double s = w * det3(Fc);
        double Gm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 0; a < NPE; ++a) {
            double La[3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
                La[k] = sdN[l][a][0] * Ji[0 * 3 + k] + sdN[l][a][1] * Ji[1 * 3 + k] +
                        sdN[l][a][2] * Ji[2 * 3 + k];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) Gm[i * 3 + k] += sl[le][a][i] * La[k];
        }
        contrib = -s * (ds[0] * Gm[0] + ds[1] * Gm[4] + ds[2] * Gm[8] +
                        ds[3] * (Gm[5] + Gm[7]) + ds[4] * (Gm[2] + Gm[6]) + ds[5] * (Gm[1] + Gm[3]));
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, off);
    if (valid && lane == 0) dJdG[e] = contrib;
}

// ---------------------------------------------------------------------------------------
// Exact directional derivative of the internal force, y = (d f_int / d u) v, by forward-mode
// differentiation (dual numbers) of the element force.  neon's assembled tangents are not the
// exact derivative of its f_int (the Kirchhoff moduli enter without 1/J, and the microsphere
// drops the -2/3 (dev tau (x) I + I (x) dev tau) term), so an adjoint that must match finite
// differences of the forward solve uses this product for its defect residual.  Hyperelastic
// and small-strain elastic models (no history): NH, microsphere, linear elasticity.
// ---------------------------------------------------------------------------------------
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)};
}
__device__ __forceinline__ Dual dlog(Dual a) { return {log(a.v), a.d / a.v}; }
__device__ __forceinline__ Dual dpow(Dual a, double p) {
    const double f = pow(a.v, p);
    return {f, p * f / a.v * a.d};
}
__device__ __forceinline__ Dual ddet3(const Dual* m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}
__device__ __forceinline__ void dinv3(const Dual* m, Dual* r) {
    const Dual c00 = m[4] * m[8] - m[5] * m[7], c10 = m[7] * m[2] - m[8] * m[1],
               c20 = m[1] * m[5] - m[2] * m[4];
    const Dual det = c00 * m[0] + c10 * m[3] + c20 * m[6];
    const Dual id = Dual{1.0, 0.0} / det;
    r[0] = c00 * id;
    r[1] = c10 * id;
    r[2] = c20 * id;
    r[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    r[4] = (m[8] * m[0] - m[6] * m[2]) * id;
    r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    r[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    r[7] = (m[6] * m[1] - m[7] * m[0]) * id;
    r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

// Cauchy stress (11 22 33 23 13 12) of the path's stateless models as a function of F, H
template <int MODEL>
__device__ __forceinline__ void dual_stress(const ElementArgs& A, double Gm, const Dual* F,
                                            const Dual* H, Dual* s) {
    if constexpr (MODEL == MODEL_LE) {
        const Dual e3 = 0.5 * (H[5] + H[7]), e4 = 0.5 * (H[2] + H[6]), e5 = 0.5 * (H[1] + H[3]);
        const Dual tr = H[0] + H[4] + H[8];
        s[0] = A.lambda * tr + 2.0 * A.G * H[0];
        s[1] = A.lambda * tr + 2.0 * A.G * H[4];
        s[2] = A.lambda * tr + 2.0 * A.G * H[8];
        s[3] = 2.0 * A.G * e3;
        s[4] = 2.0 * A.G * e4;
        s[5] = 2.0 * A.G * e5;
    } else if constexpr (MODEL == MODEL_NH) {
        const Dual J = ddet3(F);
        Dual B[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                B[i * 3 + j] = F[i * 3 + 0] * F[j * 3 + 0] + F[i * 3 + 1] * F[j * 3 + 1] +
                               F[i * 3 + 2] * F[j * 3 + 2];
        const Dual lnJ = dlog(J);
        const double mu = A.G, lam = A.lambda;
        const Dual one{1.0, 0.0};
        s[0] = (lam * lnJ + mu * (B[0] - one)) / J;
        s[1] = (lam * lnJ + mu * (B[4] - one)) / J;
        s[2] = (lam * lnJ + mu * (B[8] - one)) / J;
        s[3] = (mu * B[5]) / J;
        s[4] = (mu * B[2]) / J;
        s[5] = (mu * B[1]) / J;
    } else {
        const double K = A.K;
        const Dual J = ddet3(F);
        const Dual sc = dpow(J, -1.0 / 3.0);
        Dual acc[6] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};
        for (int i = A.sph0; i < A.sph0 + A.nsph; ++i) {
            const double r0 = c_sphere_r[3 * i], r1 = c_sphere_r[3 * i + 1],
                         r2 = c_sphere_r[3 * i + 2], w = c_sphere_w[i];
            const Dual t0 = sc * (r0 * F[0] + r1 * F[1] + r2 * F[2]);
            const Dual t1 = sc * (r0 * F[3] + r1 * F[4] + r2 * F[5]);
            const Dual t2 = sc * (r0 * F[6] + r1 * F[7] + r2 * F[8]);
            // chain weight: 3 (Gaussian) or the Pade approximant pade_first(l) (Langevin)
            Dual f{3.0, 0.0};
            if constexpr (MODEL == MODEL_ML) {
                const Dual l2 = t0 * t0 + t1 * t1 + t2 * t2;
                const Dual Nd{A.Nseg, 0.0};
                f = (3.0 * Nd - l2) / (Nd - l2);
            }
            const Dual wf = w * f;
            acc[0] = acc[0] + wf * (t0 * t0);
            acc[1] = acc[1] + wf * (t1 * t1);
            acc[2] = acc[2] + wf * (t2 * t2);
            acc[3] = acc[3] + wf * (t1 * t2);
            acc[4] = acc[4] + wf * (t0 * t2);
            acc[5] = acc[5] + wf * (t0 * t1);
        }
        Dual tau[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) tau[c] = Gm * acc[c];
        const Dual invJ = Dual{1.0, 0.0} / J;
        const Dual p = J * ((K / 2.0) * (J - invJ));
        const Dual tr3 = (1.0 / 3.0) * (tau[0] + tau[1] + tau[2]);
        s[0] = (p + tau[0] - tr3) / J;
        s[1] = (p + tau[1] - tr3) / J;
        s[2] = (p + tau[2] - tr3) / J;
        s[3] = tau[3] / J;
        s[4] = tau[4] / J;
        s[5] = tau[5] / J;
    }
}

template <int NPE, int MODEL>
__global__ void __launch_bounds__(64) k_force_jvp(ElementArgs A, const double* __restrict__ v,
                                                  double* __restrict__ y) {
    using T = Topo<NPE>;
    constexpr int NQ = T::NQ, G = T::G, EPC = T::EPC;
    __shared__ double sX[EPC][NPE][3];
    __shared__ double sx[EPC][NPE][3];
    __shared__ double sv[EPC][NPE][3];
    __shared__ double sdN[NQ][NPE][3];
    const int tid = threadIdx.x;
    const int le = tid / G;
    const int lane = tid % G;
    const long long e = (long long)blockIdx.x * EPC + le;
    const bool valid = e < A.E;
    for (int i = tid; i < NQ * NPE * 3; i += blockDim.x)
        (&sdN[0][0][0])[i] = (NPE == 8) ? c_dN_hex8[i] : c_dN_tet4[i];
    int node[(NPE + G - 1) / G];
#pragma unroll
    for (int j = 0; j < (NPE + G - 1) / G; ++j) {
        const int a = lane + j * G;
        node[j] = 0;
        if (a < NPE && valid) {
            const int nd = A.conn[e * NPE + a];
            node[j] = nd;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double Xv = A.X[3ll * nd + k];
                sX[le][a][k] = Xv;
                sx[le][a][k] = A.u[3ll * nd + k] + Xv;
                sv[le][a][k] = v[3ll * nd + k];
            }
        }
    }
    __syncthreads();
    const int l = lane;
    const bool active = valid && l < NQ;
    Dual Ji[9], s{0.0, 0.0}, sig[6];
    if (active) {
        const double w = (NPE == 8) ? c_w_hex8[l] : (1.0 / 6.0);
        Dual Fc[9], U[9];
        double F0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int i = 0; i < 9; ++i) Fc[i] = U[i] = Dual{0.0, 0.0};
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const Dual xi{sx[le][a][i], sv[le][a][i]};
                const Dual di{sx[le][a][i] - sX[le][a][i], sv[le][a][i]};
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double d = sdN[l][a][k];
                    Fc[i * 3 + k] = Fc[i * 3 + k] + d * xi;
                    U[i * 3 + k] = U[i * 3 + k] + d * di;
                    F0[i * 3 + k] += sX[le][a][i] * d;
                }
            }
        double F0i[9];
        inv3(F0, F0i);
        Dual Fd[9], Hm[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                Fd[i * 3 + j] = F0i[0 * 3 + j] * Fc[i * 3 + 0] + F0i[1 * 3 + j] * Fc[i * 3 + 1] +
                                F0i[2 * 3 + j] * Fc[i * 3 + 2];
                Hm[i * 3 + j] = F0i[0 * 3 + j] * U[i * 3 + 0] + F0i[1 * 3 + j] * U[i * 3 + 1] +
                                F0i[2 * 3 + j] * U[i * 3 + 2];
            }
        const ElementArgs Ae = element_moduli(A, e);
        dual_stress<MODEL>(Ae, Ae.G, Fd, Hm, sig);
        dinv3(Fc, Ji);
        s = w * ddet3(Fc);
    }
    double fown[(NPE + G - 1) / G][3];
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
        double g[3] = {0.0, 0.0, 0.0};
        if (active) {
            Dual La[3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
                La[k] = sdN[l][a][0] * Ji[0 * 3 + k] + sdN[l][a][1] * Ji[1 * 3 + k] +
                        sdN[l][a][2] * Ji[2 * 3 + k];
            g[0] = (s * (sig[0] * La[0] + sig[5] * La[1] + sig[4] * La[2])).d;
            g[1] = (s * (sig[5] * La[0] + sig[1] * La[1] + sig[3] * La[2])).d;
            g[2] = (s * (sig[4] * La[0] + sig[3] * La[1] + sig[2] * La[2])).d;
        }
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1)
#pragma unroll
            for (int k = 0; k < 3; ++k) g[k] += __shfl_xor_sync(0xffffffffu, g[k], off);
        if (a % G == lane)
#pragma unroll
            for (int k = 0; k < 3; ++k) fown[a / G][k] = g[k];
    }
    if (!valid) return;
#pragma unroll
    for (int j = 0; j < (NPE + G - 1) / G; ++j) {
        const int a = lane + j * G;
        if (a < NPE)
#pragma unroll
            for (int k = 0; k < 3; ++k) atomicAdd(&y[3ll * node[j] + k], fown[j][k]);
    }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
static bool g_tables_ready = false;

static int upload_tables(nb2_ctx* c) {
    if (g_tables_ready) return NB2_OK;
    // hexahedron8 shape derivatives at the 8-point rule (hexahedron.cpp:10-67,
    // hexahedron_quadrature.cpp:27-40)
    const double lc[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                             {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    const double g = 1.0 / std::sqrt(3.0);
    const double qc[8][3] = {{-g, -g, -g}, {g, -g, -g}, {g, g, -g}, {-g, g, -g},
                             {-g, -g, g},  {g, -g, g},  {g, g, g},  {-g, g, g}};
    double dN[8 * 8 * 3], w[8];
    for (int l = 0; l < 8; ++l) {
        w[l] = 1.0;
        for (int a = 0; a < 8; ++a) {
            double xa = lc[a][0], ea = lc[a][1], za = lc[a][2];
            double xi = qc[l][0], eta = qc[l][1], zeta = qc[l][2];
            dN[(l * 8 + a) * 3 + 0] = 1.0 / 8.0 * xa * (1.0 + ea * eta) * (1.0 + za * zeta);
            dN[(l * 8 + a) * 3 + 1] = 1.0 / 8.0 * (1.0 + xa * xi) * ea * (1.0 + za * zeta);
            dN[(l * 8 + a) * 3 + 2] = 1.0 / 8.0 * (1.0 + xa * xi) * (1.0 + ea * eta) * za;
        }
    }
    // tetrahedron4 (tetrahedron.cpp:6-45)
    const double dNt[12] = {1, 0, 0, 0, 1, 0, 0, 0, 1, -1, -1, -1};
    // BO21 (unit_sphere_quadrature.cpp:10-31)
    const double w1 = 0.0265214244093 * 2.0, w2 = 0.0199301476312 * 2.0, w3 = 0.0250712367487 * 2.0;
    const double d0 = 0.707106781187, d1 = 0.387907304067, d2 = 0.836095596749;
    const double r[21 * 3] = {1, 0, 0, 0, 1, 0, 0, 0, 1, d0, d0, 0, d0, -d0, 0, d0, 0, d0, d0, 0, -d0,
                              0, d0, d0, 0, d0, -d0, d1, d1, d2, d1, d1, -d2, d1, -d1, d2, d1, -d1,
                              -d2, d1, d2, d1, d1, d2, -d1, d1, -d2, d1, d1, -d2, -d1, d2, d1, d1,
                              d2, d1, -d1, d2, -d1, d1, d2, -d1, -d1};
    // BO33 (unit_sphere_quadrature.cpp:33-91), after BO21 in the same tables
    const double v1 = 2.0 * 0.00985353993433, v2 = 2.0 * 0.0162969685886,
                 v3 = 2.0 * 0.0134788844008, v4 = 2.0 * 0.0175759129880;
    const double a = 0.707106781187, b = 0.933898956394, cc = 0.357537045978,
                 d = 0.437263676092, ee = 0.785875915868;
    const double r33[33 * 3] = {1, 0, 0, 0, 1, 0, 0, 0, 1,
                                a, a, 0, a, -a, 0, a, 0, a, a, 0, -a, 0, a, a, 0, a, -a,
                                b, cc, 0, b, -cc, 0, cc, b, 0, cc, -b, 0,
                                b, 0, cc, b, 0, -cc, cc, 0, b, cc, 0, -b,
                                0, b, cc, 0, b, -cc, 0, cc, b, 0, cc, -b,
                                d, d, ee, d, d, -ee, d, -d, ee, d, -d, -ee,
                                d, ee, d, d, ee, -d, d, -ee, d, d, -ee, -d,
                                ee, d, d, ee, d, -d, ee, -d, d, ee, -d, -d};
    double rr[(21 + 33) * 3], sw[21 + 33];
    for (int i = 0; i < 21 * 3; ++i) rr[i] = r[i];
    for (int i = 0; i < 33 * 3; ++i) rr[21 * 3 + i] = r33[i];
    for (int i = 0; i < 21; ++i) sw[i] = i < 3 ? w1 : (i < 9 ? w2 : w3);
    for (int i = 0; i < 33; ++i) sw[21 + i] = i < 3 ? v1 : (i < 9 ? v2 : (i < 21 ? v3 : v4));
    NB2_CUDA(c, cudaMemcpyToSymbol(c_dN_hex8, dN, sizeof dN));
    NB2_CUDA(c, cudaMemcpyToSymbol(c_w_hex8, w, sizeof w));
    NB2_CUDA(c, cudaMemcpyToSymbol(c_hex8_g, &g, sizeof g));
    NB2_CUDA(c, cudaMemcpyToSymbol(c_dN_tet4, dNt, sizeof dNt));
    NB2_CUDA(c, cudaMemcpyToSymbol(c_sphere_r, rr, sizeof rr));
    NB2_CUDA(c, cudaMemcpyToSymbol(c_sphere_w, sw, sizeof sw));
    float dNf[8 * 8 * 3], dNtf[12];
    for (int i = 0; i < 8 * 8 * 3; ++i) dNf[i] = (float)dN[i];
    for (int i = 0; i < 12; ++i) dNtf[i] = (float)dNt[i];
    NB2_CUDA(c, cudaMemcpyToSymbol(c_dNf_hex8, dNf, sizeof dNf));
    NB2_CUDA(c, cudaMemcpyToSymbol(c_dNf_tet4, dNtf, sizeof dNtf));
    g_tables_ready = true;
    return NB2_OK;
}

// elements a launch covers: the launch's colour in a colour-partitioned pass, else all
static unsigned launch_elements(const nb2_ctx*, const ElementArgs& A) {
    return (unsigned)A.ecount;
}

template <int NPE, int MODEL, typename Real, int MODE>
static void launch_one(nb2_ctx* c, const ElementArgs& A) {
    constexpr int EPC = Topo<NPE>::EPC, G = Topo<NPE>::G;
    const unsigned grid = (launch_elements(c, A) + EPC - 1) / EPC;
    if (grid == 0) return;
    k_element<NPE, MODEL, Real, MODE><<<grid, EPC * G, 0, c->stream>>>(A);
    c->launches++;
}

template <int NPE, int MODEL>
static int dispatch_mode(nb2_ctx* c, const ElementArgs& A, int mode, int precision) {
    constexpr int FUSED = MODE_CONSTITUTIVE | MODE_STIFFNESS | MODE_FORCE;
    constexpr int RESID = MODE_CONSTITUTIVE | MODE_FORCE;
    constexpr int UPD = MODE_CONSTITUTIVE | MODE_STORE;
    constexpr int ASM = MODE_STIFFNESS | MODE_FORCE;
    constexpr int FUSED_STORE = FUSED | MODE_STORE;
    if (mode == FUSED && precision == NB2_FP64) launch_one<NPE, MODEL, double, FUSED>(c, A);
    else if (mode == FUSED) launch_one<NPE, MODEL, float, FUSED>(c, A);
    else if (mode == FUSED_STORE && precision != NB2_FP64)
        launch_one<NPE, MODEL, float, FUSED_STORE>(c, A);
    else if (mode == (RESID | MODE_STORE)) launch_one<NPE, MODEL, double, RESID | MODE_STORE>(c, A);
    else if (mode == RESID) launch_one<NPE, MODEL, double, RESID>(c, A);
    else if (mode == UPD) launch_one<NPE, MODEL, double, UPD>(c, A);
    else if (mode == ASM) launch_one<NPE, MODEL, double, ASM>(c, A);
    else return NB2_E_INPUT;
    return NB2_OK;
}

template <int NPE>
static int dispatch_model(nb2_ctx* c, const ElementArgs& A, int mode, int precision) {
    switch (c->mat.model) {
        case MODEL_LE: return dispatch_mode<NPE, MODEL_LE>(c, A, mode, precision);
        case MODEL_NH: return dispatch_mode<NPE, MODEL_NH>(c, A, mode, precision);
        case MODEL_J2: return dispatch_mode<NPE, MODEL_J2>(c, A, mode, precision);
        case MODEL_MS: return dispatch_mode<NPE, MODEL_MS>(c, A, mode, precision);
        case MODEL_ML: return dispatch_mode<NPE, MODEL_ML>(c, A, mode, precision);
        case MODEL_MN: return dispatch_mode<NPE, MODEL_MN>(c, A, mode, precision);
    }
    return NB2_E_INPUT;
}

static ElementArgs make_args(nb2_ctx* c);
static bool colour_applies(const nb2_ctx* c, int mode, int precision);


template <int NPE>
static void launch_apply_t(nb2_ctx* c, const ElementArgs& A, const double* v, double* y) {
    constexpr int EPC = Topo<NPE>::EPC, G = Topo<NPE>::G;
    const unsigned grid = (launch_elements(c, A) + EPC - 1) / EPC;
    if (grid == 0) return;
    switch (c->mat.model) {
        case MODEL_LE: k_apply<NPE, MODEL_LE><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
        case MODEL_NH: k_apply<NPE, MODEL_NH><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
        case MODEL_J2: k_apply<NPE, MODEL_J2><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
        case MODEL_ML: k_apply<NPE, MODEL_ML><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
        case MODEL_MN: k_apply<NPE, MODEL_MN><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
        default: k_apply<NPE, MODEL_MS><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
    }
    c->launches++;
}

// y = K v (FP64, matrix-free) with the tangent stored by the last MODE_STORE pass
int launch_apply(nb2_ctx* c, const double* v, double* y) {
    int st = upload_tables(c);
    if (st) return st;
    if (!c->dpar || !c->u_tan) return NB2_E_INPUT;
    bool coloured = false;
    if (colour_applies(c, MODE_FORCE, NB2_FP64)) {
        NB2_TRY(ensure_colouring(c));
        coloured = c->colour_state == 1;
    }
    ElementArgs A = make_args(c);
    A.u = c->u_tan;
    NB2_CUDA(c, cudaMemsetAsync(y, 0, sizeof(double) * c->n, c->stream));
    if (coloured) {
        // one launch per colour: each entry gets at most one term per launch, in colour order
        for (size_t k = 0; k + 1 < c->h_coff.size(); ++k) {
            A.order = c->corder + c->h_coff[k];
            A.ecount = c->h_coff[k + 1] - c->h_coff[k];
            launch_apply_t<8>(c, A, v, y);
        }
    } else if (c->npe == 8) {
        launch_apply_t<8>(c, A, v, y);
    } else {
        launch_apply_t<4>(c, A, v, y);
    }
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

template <int NPE>
static void element_stiffness_t(nb2_ctx* c, const ElementArgs& A, long long e, double* Ke) {
    switch (c->mat.model) {
        case MODEL_LE: k_element_stiffness<NPE, MODEL_LE><<<1, 32, 0, c->stream>>>(A, e, Ke); break;
        case MODEL_NH: k_element_stiffness<NPE, MODEL_NH><<<1, 32, 0, c->stream>>>(A, e, Ke); break;
        case MODEL_J2: k_element_stiffness<NPE, MODEL_J2><<<1, 32, 0, c->stream>>>(A, e, Ke); break;
        case MODEL_ML: k_element_stiffness<NPE, MODEL_ML><<<1, 32, 0, c->stream>>>(A, e, Ke); break;
        case MODEL_MN: k_element_stiffness<NPE, MODEL_MN><<<1, 32, 0, c->stream>>>(A, e, Ke); break;
        default: k_element_stiffness<NPE, MODEL_MS><<<1, 32, 0, c->stream>>>(A, e, Ke); break;
    }
    c->launches++;
}

// Ke_dev [3 npe][3 npe] = element e's tangent stiffness from the tangent stored by the last
// MODE_STORE pass
int launch_element_stiffness(nb2_ctx* c, long long e, double* Ke_dev) {
    int st = upload_tables(c);
    if (st) return st;
    if (!c->dpar || !c->u_tan || e < 0 || e >= c->E) return NB2_E_INPUT;
    ElementArgs A = make_args(c);
    A.u = c->u_tan;
    if (c->npe == 8)
        element_stiffness_t<8>(c, A, e, Ke_dev);
    else
        element_stiffness_t<4>(c, A, e, Ke_dev);
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

template <int NPE, int MODEL>
static void mf_setup_t(nb2_ctx* c, const ElementArgs& A) {
    constexpr int EPC = Topo<NPE>::EPC, G = Topo<NPE>::G;
    const unsigned grid = (unsigned)((c->E + EPC - 1) / EPC);
    k_mf_setup<NPE, MODEL><<<grid, EPC * G, 0, c->stream>>>(A, c->mf_d, c->mf_c, c->mf_ye);
    c->launches++;
}

// FP32 matrix-free data of the tangent stored by the last MODE_STORE pass; the element
// contributions to diag(K) are left in mf_ye for the gather that forms the Jacobi inverse
int launch_mf_setup(nb2_ctx* c) {
    int st = upload_tables(c);
    if (st) return st;
    if (!c->dpar || !c->u_tan || !c->mf_d) return NB2_E_INPUT;
    ElementArgs A = make_args(c);
    A.u = c->u_tan;
    const bool hex = c->npe == 8;
    switch (c->mat.model) {
        case MODEL_LE: hex ? mf_setup_t<8, MODEL_LE>(c, A) : mf_setup_t<4, MODEL_LE>(c, A); break;
        case MODEL_NH: hex ? mf_setup_t<8, MODEL_NH>(c, A) : mf_setup_t<4, MODEL_NH>(c, A); break;
        case MODEL_J2: hex ? mf_setup_t<8, MODEL_J2>(c, A) : mf_setup_t<4, MODEL_J2>(c, A); break;
        case MODEL_ML: hex ? mf_setup_t<8, MODEL_ML>(c, A) : mf_setup_t<4, MODEL_ML>(c, A); break;
        case MODEL_MN: hex ? mf_setup_t<8, MODEL_MN>(c, A) : mf_setup_t<4, MODEL_MN>(c, A); break;
        default: hex ? mf_setup_t<8, MODEL_MS>(c, A) : mf_setup_t<4, MODEL_MS>(c, A); break;
    }
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

int mf_coefficients(int model) {
    switch (model) {
        case MODEL_LE: return MfCoef<MODEL_LE>::KC;
        case MODEL_NH: return MfCoef<MODEL_NH>::KC;
        case MODEL_J2: return MfCoef<MODEL_J2>::KC;
        case MODEL_ML: return MfCoef<MODEL_ML>::KC;
        case MODEL_MN: return MfCoef<MODEL_MN>::KC;
        default: return MfCoef<MODEL_MS>::KC;
    }
}

template <int NPE, int MODEL>
static void apply32_t(nb2_ctx* c, const float* v, float* ye, const int* done) {
    const unsigned grid = (unsigned)((c->E + kApply32Threads - 1) / kApply32Threads);
    k_apply32<NPE, MODEL><<<grid, kApply32Threads, 0, c->stream>>>(
        c->E, c->conn, c->mf_d, c->mf_c, c->nqp, (float)c->mat.bulk_modulus, v, ye, done);
}

// ye = K_e v_e per element in FP32 (graph-capturable: launches only)
void enqueue_apply32(nb2_ctx* c, const float* v, float* ye, const int* done) {
    const bool hex = c->npe == 8;
    switch (c->mat.model) {
        case MODEL_LE: hex ? apply32_t<8, MODEL_LE>(c, v, ye, done) : apply32_t<4, MODEL_LE>(c, v, ye, done); break;
        case MODEL_NH: hex ? apply32_t<8, MODEL_NH>(c, v, ye, done) : apply32_t<4, MODEL_NH>(c, v, ye, done); break;
        case MODEL_J2: hex ? apply32_t<8, MODEL_J2>(c, v, ye, done) : apply32_t<4, MODEL_J2>(c, v, ye, done); break;
        case MODEL_ML: hex ? apply32_t<8, MODEL_ML>(c, v, ye, done) : apply32_t<4, MODEL_ML>(c, v, ye, done); break;
        case MODEL_MN: hex ? apply32_t<8, MODEL_MN>(c, v, ye, done) : apply32_t<4, MODEL_MN>(c, v, ye, done); break;
        default: hex ? apply32_t<8, MODEL_MS>(c, v, ye, done) : apply32_t<4, MODEL_MS>(c, v, ye, done); break;
    }
}

template <int NPE>
static int launch_jvp_t(nb2_ctx* c, const ElementArgs& A, const double* v, double* y) {
    constexpr int EPC = Topo<NPE>::EPC, G = Topo<NPE>::G;
    const unsigned grid = (unsigned)((c->E + EPC - 1) / EPC);
    switch (c->mat.model) {
        case MODEL_LE: k_force_jvp<NPE, MODEL_LE><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
        case MODEL_NH: k_force_jvp<NPE, MODEL_NH><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
        case MODEL_MS: k_force_jvp<NPE, MODEL_MS><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
        case MODEL_ML: k_force_jvp<NPE, MODEL_ML><<<grid, EPC * G, 0, c->stream>>>(A, v, y); break;
        default: return NB2_E_INPUT;  // J2 carries history; the non-affine model has no product here
    }
    c->launches++;
    return NB2_OK;
}

// y = (d f_int / d u) v exactly (forward-mode), at the context displacement
int launch_force_jvp(nb2_ctx* c, const double* v, double* y) {
    int st = upload_tables(c);
    if (st) return st;
    ElementArgs A = make_args(c);
    NB2_CUDA(c, cudaMemsetAsync(y, 0, sizeof(double) * c->n, c->stream));
    st = c->npe == 8 ? launch_jvp_t<8>(c, A, v, y) : launch_jvp_t<4>(c, A, v, y);
    if (st) return st;
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

int launch_adjoint_shear(nb2_ctx* c, const double* lam, double* dJdG) {
    int st = upload_tables(c);
    if (st) return st;
    ElementArgs A = make_args(c);
    const bool lgv = c->mat.model == MODEL_ML;
    if (c->npe == 8) {
        constexpr int EPC = Topo<8>::EPC, G = Topo<8>::G;
        const unsigned grid = (unsigned)((c->E + EPC - 1) / EPC);
        if (lgv)
            k_adjoint_shear<8, MODEL_ML><<<grid, EPC * G, 0, c->stream>>>(A, lam, dJdG);
        else
            k_adjoint_shear<8, MODEL_MS><<<grid, EPC * G, 0, c->stream>>>(A, lam, dJdG);
    } else {
        constexpr int EPC = Topo<4>::EPC, G = Topo<4>::G;
        const unsigned grid = (unsigned)((c->E + EPC - 1) / EPC);
        if (lgv)
            k_adjoint_shear<4, MODEL_ML><<<grid, EPC * G, 0, c->stream>>>(A, lam, dJdG);
        else
            k_adjoint_shear<4, MODEL_MS><<<grid, EPC * G, 0, c->stream>>>(A, lam, dJdG);
    }
    c->launches++;
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

static ElementArgs make_args(nb2_ctx* c) {
    ElementArgs A;
    A.X = c->X;
    A.u = c->u;
    A.conn = c->conn;
    A.slot = c->slot;
    A.E = c->E;
    A.nqp = c->nqp;
    A.K = c->mat.bulk_modulus;
    A.G = c->mat.shear_modulus;
    A.lambda = c->mat.bulk_modulus - 2.0 * c->mat.shear_modulus / 3.0;
    A.sigma_y = c->mat.yield_stress;
    A.H_iso = c->mat.isotropic_hardening_modulus;
    A.Nseg = c->mat.segments_per_chain;
    A.p_na = c->mat.nonaffine_stretch_parameter;
    A.sph0 = c->mat.unit_sphere_points == 33 ? 21 : 0;
    A.nsph = c->mat.unit_sphere_points == 33 ? 33 : 21;
    A.Ge = c->Ge;
    A.Ke = c->Ke;
    A.ep = c->ep;
    A.epbar = c->epbar;
    A.K64 = c->K64;
    A.K32 = c->K32;
    A.fint = c->fint;
    A.sig = c->sig;
    A.dpar = c->dpar;
    A.detF = c->detF;
    A.status = c->status;
    A.e_inst = c->e_inst;
    A.inst_on = c->inst_on;
    A.inst_flags = c->inst_flags;
    A.order = nullptr;  // colour-partitioned passes set these per launch
    A.ecount = c->E;
    return A;
}

// The colour-partitioned launches (NB2_SCATTER_COLOURED, and always inside nb2_static_solve)
// serve hex8 passes of one problem that scatter f_int, with the stiffness only in FP64 on the mma
// path (not the anisotropic microsphere tangent); batched instances (element gating), tet4 and
// FP32 K use one launch.
static bool colour_applies(const nb2_ctx* c, int mode, int precision) {
    if (c->scatter != NB2_SCATTER_COLOURED && !c->newton_scatter) return false;
    if (c->npe != 8 || c->e_inst || !(mode & MODE_FORCE)) return false;
    if (mode & MODE_STIFFNESS) return precision == NB2_FP64 && !model_aniso(c->mat.model);
    return true;
}

int launch_element_kernel(nb2_ctx* c, int mode, int precision) {
    int st = upload_tables(c);
    if (st) return st;
    bool coloured = false;
    if (colour_applies(c, mode, precision)) {
        NB2_TRY(ensure_colouring(c));
        coloured = c->colour_state == 1;
    }
    // FP64 K of one problem is double-buffered: the buffer zeroed in the background during the
    // previous pass becomes K, and the previous K is zeroed during this pass (it is no longer
    // read once the work queued before this pass is done)
    const bool kdouble = (mode & MODE_STIFFNESS) && precision == NB2_FP64 && !c->e_inst;
    if (kdouble) NB2_TRY(ensure_k64_alt(c));
    const bool kbg = kdouble && c->kalt_state == 1;
    if (mode & MODE_STIFFNESS) {
        if (kbg && c->alt_zeroed) {
            std::swap(c->K64, c->K64_alt);
            c->kbuf ^= 1;
            NB2_CUDA(c, cudaStreamWaitEvent(c->stream, c->zev_done, 0));
            c->alt_zeroed = false;
        } else if (precision == NB2_FP64) {
            NB2_CUDA(c, cudaMemsetAsync(c->K64, 0, sizeof(double) * 9 * c->nnzb, c->stream));
        } else {
            NB2_CUDA(c, cudaMemsetAsync(c->K32, 0, sizeof(float) * 9 * c->nnzb, c->stream));
        }
    }
    if (kbg) {
        NB2_CUDA(c, cudaEventRecord(c->zev_free, c->stream));
        NB2_CUDA(c, cudaStreamWaitEvent(c->zstream, c->zev_free, 0));
    }
    ElementArgs A = make_args(c);
    if (mode & MODE_FORCE) NB2_CUDA(c, cudaMemsetAsync(c->fint, 0, sizeof(double) * c->n, c->stream));
    if (coloured) {
        // one launch per colour: an entry of K or f_int receives at most one term per launch,
        // so its additions arrive in colour order on every run
        for (size_t k = 0; k + 1 < c->h_coff.size(); ++k) {
            A.order = c->corder + c->h_coff[k];
            A.ecount = c->h_coff[k + 1] - c->h_coff[k];
            st = dispatch_model<8>(c, A, mode, precision);
            if (st) return st;
        }
    } else {
        st = (c->npe == 8) ? dispatch_model<8>(c, A, mode, precision)
                           : dispatch_model<4>(c, A, mode, precision);
        if (st) return st;
    }
    if (kbg) {
        NB2_CUDA(c, cudaMemsetAsync(c->K64_alt, 0, sizeof(double) * 9 * c->nnzb, c->zstream));
        NB2_CUDA(c, cudaEventRecord(c->zev_done, c->zstream));
        c->alt_zeroed = true;
    }
    // the matrix-free tangent re-derives the gradients from this displacement, not from a
    // later one (the Newton step adds the prescribed increment before its first solve)
    if ((mode & MODE_STORE) && c->u_tan)
        NB2_CUDA(c, cudaMemcpyAsync(c->u_tan, c->u, sizeof(double) * c->n,
                                    cudaMemcpyDeviceToDevice, c->stream));
    NB2_CUDA(c, cudaGetLastError());
    return NB2_OK;
}

// Canonical algorithmic FLOPs per element (hex8 small strain 29,040; hex8 finite strain 32,240;
// tet4 finite strain 1,552) plus the constitutive update per point (LE 60, NH 120, J2 250,
// microsphere BO21 2,000, Langevin microsphere BO21 3,000, non-affine BO21 4,500); the
// anisotropic tangent of the Langevin and non-affine models
// adds 81 FMAs per block and point (hex8 36 blocks x 8 points, tet4 10 x 1).
void element_flop_model(const nb2_ctx* c, double* flops_per_element) {
    double base;
    bool finite = c->mat.model == MODEL_NH || c->mat.model == MODEL_MS ||
                  model_aniso(c->mat.model);
    if (c->npe == 8)
        base = finite ? 32240.0 : 29040.0;
    else
        base = 1552.0;
    if (model_aniso(c->mat.model)) base += 2.0 * 81.0 * (c->npe == 8 ? 36 * 8 : 10);
    const double cm[6] = {60.0, 120.0, 250.0, 2000.0, 3000.0, 4500.0};
    *flops_per_element = base + c->nq * cm[c->mat.model];
}

}  // namespace nb2
