// mf_kernels.cuh -- the FP32 matrix-free tangent product of the mixed-precision PCG (included
// by elements.cu, which owns the shape-function tables).
//
// The assembled FP32 K of a hex8 mesh costs ~27 blocks x 40 B = 1.1 KB per element per SpMV.
// The same operator applied element by element needs far less: per element the FP32 node
// coordinates relative to its first node (96 B; differences taken in FP64, so no cancellation
// in FP32), per quadrature point the tangent coefficients pre-multiplied by w det J (2 floats;
// J2 plastic points 9, finite strain 8, anisotropic microspheres 8 + 21), the node indices, the
// input/output vectors.
//   k_mf_setup  once per linear solve (after an element pass that stored its outputs): writes
//               those FP32 data and each element's contribution to diag(K) (Jacobi);
//   k_apply32   per CG iteration: y_e = K_e v_e in FP32, written per local node plane
//               (ye[npe][E][3]);
//               a node-ordered gather (pcg.cu) sums ye into q without atomics, in a fixed order.
// With G = sum_b v_b (x) L_b the element force of node a is (the product the assembled blocks
//   K_ab = s[lam' La(x)Lb + mu'((La.Lb) I + Lb(x)La) + b (N La)(x)(N Lb)] + s (La.sigma.Lb) I
// give) y_a = s [lam' tr(G) La + mu' (G + G^T) La + b (N:G) N La + (Da eps(G)) La + G sigma La].
#pragma once

__device__ __forceinline__ float det3f(const float* m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// r = m^-1; returns det m
__device__ __forceinline__ float inv3f(const float* m, float* r) {
    const float c00 = m[4] * m[8] - m[5] * m[7];
    const float c10 = m[7] * m[2] - m[8] * m[1];
    const float c20 = m[1] * m[5] - m[2] * m[4];
    const float det = c00 * m[0] + c10 * m[3] + c20 * m[6];
    const float id = 1.0f / det;
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

// number of FP32 coefficients per quadrature point
template <int MODEL>
struct MfCoef {
    static constexpr int KC =
        (MODEL == MODEL_J2) ? 6 : ((MODEL == MODEL_LE) ? 2 : (model_aniso(MODEL) ? 8 + 21 : 8));
};

// Setup from the stored FP64 outputs of the last MODE_STORE pass (A.u = its displacement):
//   md[e][3a+k]  = (float)(x_a - x_0)_k
//   mc[c][q]     = s lam', s mu' | finite strain: then s sigma (6)
//                  | Langevin / non-affine microsphere: then s Da (21, packed upper triangle)
//                  | J2: mu' (negated at a plastic point), m = sqrt(-b) N as its 11 22 23 13 12
//                    components (N is deviatoric, so m_33 = -m_11 - m_22).  The J2 tangent is
//                    lam' I(x)I + 2 mu' I + b N(x)N with lam' = K - 2 mu'/3, and b < 0 at a
//                    plastic point (b = -6 G^2 sigma_y(ebar) / (q_trial (3G + H)) for the linear
//                    hardening return map), so b N(x)N = -m(x)m.  The point weight s = w det J
//                    comes from the element's own FP32 geometry at apply time.  Six numbers per
//                    point instead of nine, one at an elastic point.  (Were b ever positive, the
//                    operator would drop that term: the FP64 residual replacements still
//                    converge, only more slowly.)
//   de[a][e][i]  = element contribution to K_(3a+i, 3a+i) (the per-node planes of ye)
template <int NPE, int MODEL>
__global__ void __launch_bounds__(64) k_mf_setup(ElementArgs A, float* __restrict__ md,
                                                 float* __restrict__ mc, float* __restrict__ de) {
    using T = Topo<NPE>;
    constexpr int NQ = T::NQ, G = T::G, EPC = T::EPC;
    constexpr bool kFinite = (MODEL == MODEL_NH || MODEL == MODEL_MS || model_aniso(MODEL));
    constexpr bool kJ2 = (MODEL == MODEL_J2);
    constexpr bool kAniso = model_aniso(MODEL);
    __shared__ double sx[EPC][NPE][3];
    __shared__ double sdN[NQ][NPE][3];
    __shared__ double sD[EPC][NQ][NPE * 3];
    const int tid = threadIdx.x;
    const int le = tid / G;
    const int lane = tid % G;
    const long long e = (long long)blockIdx.x * EPC + le;
    const bool valid = element_enabled(A, e);
    for (int i = tid; i < NQ * NPE * 3; i += blockDim.x)
        (&sdN[0][0][0])[i] = (NPE == 8) ? c_dN_hex8[i] : c_dN_tet4[i];
#pragma unroll
    for (int j = 0; j < (NPE + G - 1) / G; ++j) {
        const int a = lane + j * G;
        if (a < NPE && valid) {
            const int nd = A.conn[e * NPE + a];
#pragma unroll
            for (int k = 0; k < 3; ++k) sx[le][a][k] = A.u[3ll * nd + k] + A.X[3ll * nd + k];
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < (NPE + G - 1) / G; ++j) {
        const int a = lane + j * G;
        if (a < NPE && valid)
#pragma unroll
            for (int k = 0; k < 3; ++k)
                md[e * NPE * 3 + 3 * a + k] = (float)(sx[le][a][k] - sx[le][0][k]);
    }
    for (int l = lane; l < NQ; l += G) {
        if (!valid) break;
        const double w = (NPE == 8) ? c_w_hex8[l] : (1.0 / 6.0);
        const long long q = e * NQ + l;
        const long long n = A.nqp;
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
        const double lam = A.dpar[0 * n + q], mu = A.dpar[1 * n + q];
        double b = 0.0, N6[6] = {0, 0, 0, 0, 0, 0}, sg[6] = {0, 0, 0, 0, 0, 0};
        if constexpr (kJ2) {
            b = A.dpar[2 * n + q];
#pragma unroll
            for (int c = 0; c < 6; ++c) N6[c] = A.dpar[(3 + c) * n + q];
            const bool plastic = b != 0.0;
            mc[0 * n + q] = plastic ? -(float)fmax(mu, 1e-30) : (float)mu;
            const double sb = plastic ? sqrt(fmax(-b, 0.0)) : 0.0;
            mc[1 * n + q] = (float)(sb * N6[0]);
            mc[2 * n + q] = (float)(sb * N6[1]);
            mc[3 * n + q] = (float)(sb * N6[3]);
            mc[4 * n + q] = (float)(sb * N6[4]);
            mc[5 * n + q] = (float)(sb * N6[5]);
        } else {
            mc[0 * n + q] = (float)(s * lam);
            mc[1 * n + q] = (float)(s * mu);
        }
        if constexpr (kFinite) {
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                sg[c] = A.sig[c * n + q];
                mc[(2 + c) * n + q] = (float)(s * sg[c]);
            }
        }
        double Da[kAniso ? 21 : 1];
        if constexpr (kAniso) {
#pragma unroll
            for (int c = 0; c < 21; ++c) {
                Da[c] = A.dpar[(3 + c) * n + q];
                mc[(8 + c) * n + q] = (float)(s * Da[c]);
            }
        }
#pragma unroll
        for (int a = 0; a < NPE; ++a) {
            double La[3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
                La[k] = sdN[l][a][0] * Ji[0 * 3 + k] + sdN[l][a][1] * Ji[1 * 3 + k] +
                        sdN[l][a][2] * Ji[2 * 3 + k];
            const double LL = La[0] * La[0] + La[1] * La[1] + La[2] * La[2];
            double nl[3] = {0, 0, 0};
            if constexpr (kJ2) {
                nl[0] = N6[0] * La[0] + N6[5] * La[1] + N6[4] * La[2];
                nl[1] = N6[5] * La[0] + N6[1] * La[1] + N6[3] * La[2];
                nl[2] = N6[4] * La[0] + N6[3] * La[1] + N6[2] * La[2];
            }
            double geo = 0.0;
            if constexpr (kFinite)
                geo = sg[0] * La[0] * La[0] + sg[1] * La[1] * La[1] + sg[2] * La[2] * La[2] +
                      2.0 * (sg[3] * La[1] * La[2] + sg[4] * La[0] * La[2] + sg[5] * La[0] * La[1]);
            double ka[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            if constexpr (kAniso) aniso_block(Da, La, La, ka);
#pragma unroll
            for (int i = 0; i < 3; ++i)
                sD[le][l][3 * a + i] = s * (lam * La[i] * La[i] + mu * (LL + La[i] * La[i]) +
                                            b * nl[i] * nl[i] + geo + ka[4 * i]);
        }
    }
    __syncthreads();
    if (!valid) return;
#pragma unroll
    for (int j = 0; j < (NPE + G - 1) / G; ++j) {
        const int a = lane + j * G;
        if (a < NPE)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                double t = 0.0;
#pragma unroll
                for (int l = 0; l < NQ; ++l) t += sD[le][l][3 * a + i];
                de[((long long)a * A.E + e) * 3 + i] = (float)t;
            }
    }
}

// ye[e] = K_e v_e in FP32 from the setup data; skipped once the CG scalars say done.
// One thread per element: its relative coordinates, input values and output stay in registers,
// so the hot loops are FFMA only.  Per point, with J = sum_a d_a (x) dN_a, Gx = sum_a v_a (x) dN_a:
//   G = Gx J^-1,  S = s[lam' tr(G) I + mu' (G + G^T) + b (N:G) N + G sigma],  P = S J^-T,
//   y_a += P dN_a                     (y_a = S L_a with L_a = J^-T dN_a, never formed)
// hex8 works in the element's trilinear modes (1, xi, eta, zeta, xi eta, xi zeta, eta zeta,
// xi eta zeta): a +/- butterfly turns the 8 nodal vectors into modal coefficients, the reference
// gradient at a point is then 4 terms per entry, and the outputs are accumulated per mode and
// turned back into nodal forces once -- about 30% fewer FMAs than nodal sums at every point.
// (The factor 1/8 of the trilinear shape functions cancels: J and Gx carry it alike, and
// P dN_a carries 8 * 1/8.)
constexpr int kApply32Threads = 128;

template <int NPE>
__device__ __forceinline__ float dNf(int i) {
    if constexpr (NPE == 8)
        return c_dNf_hex8[i];
    else
        return c_dNf_tet4[i];
}

// P = S J^-T at one point (J, Gx as defined above, in the same scaling).  J2 only: kdet turns
// det J into the point weight s (w times the determinant of the true Jacobian), Kb is the bulk
// modulus.
template <int MODEL>
__device__ __forceinline__ void point_flux(const float* J, const float* Gx,
                                           const float* __restrict__ mc, long long nqp,
                                           long long q, float kdet, float Kb, float* Pm) {
    constexpr bool kFinite = (MODEL == MODEL_NH || MODEL == MODEL_MS || model_aniso(MODEL));
    constexpr bool kJ2 = (MODEL == MODEL_J2);
    float Ji[9];
    const float det = inv3f(J, Ji);
    float G[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            G[i * 3 + k] = Gx[i * 3 + 0] * Ji[0 * 3 + k] + Gx[i * 3 + 1] * Ji[1 * 3 + k] +
                           Gx[i * 3 + 2] * Ji[2 * 3 + k];
    float cl, cm, c0 = 0.0f, sw = 0.0f;
    if constexpr (kJ2) {
        c0 = mc[0 * nqp + q];
        const float mu = fabsf(c0);
        sw = det * kdet;
        cm = sw * mu;
        cl = sw * (Kb - (2.0f / 3.0f) * mu);
    } else {
        cl = mc[0 * nqp + q];
        cm = mc[1 * nqp + q];
    }
    const float ltr = cl * (G[0] + G[4] + G[8]);
    float S[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            S[i * 3 + k] = cm * (G[i * 3 + k] + G[k * 3 + i]) + (i == k ? ltr : 0.0f);
    if constexpr (kJ2) {
        if (c0 < 0.0f) {  // plastic point: S -= s (m:G) m
            const float m0 = mc[1 * nqp + q], m1 = mc[2 * nqp + q], m3 = mc[3 * nqp + q],
                        m4 = mc[4 * nqp + q], m5 = mc[5 * nqp + q];
            const float m2 = -(m0 + m1);
            const float bN = -sw * (m0 * G[0] + m1 * G[4] + m2 * G[8] + m3 * (G[5] + G[7]) +
                                    m4 * (G[2] + G[6]) + m5 * (G[1] + G[3]));
            // m symmetric (11 22 33 23 13 12)
            S[0] += bN * m0; S[4] += bN * m1; S[8] += bN * m2;
            S[5] += bN * m3; S[7] += bN * m3;
            S[2] += bN * m4; S[6] += bN * m4;
            S[1] += bN * m5; S[3] += bN * m5;
        }
    }
    if constexpr (model_aniso(MODEL)) {
        float Da[21], sa[6];
#pragma unroll
        for (int c = 0; c < 21; ++c) Da[c] = mc[(8 + c) * nqp + q];
        aniso_stress(Da, G, sa);
        S[0] += sa[0]; S[4] += sa[1]; S[8] += sa[2];
        S[5] += sa[3]; S[7] += sa[3];
        S[2] += sa[4]; S[6] += sa[4];
        S[1] += sa[5]; S[3] += sa[5];
    }
    if constexpr (kFinite) {
        float sg[9];
        sg[0] = mc[2 * nqp + q]; sg[4] = mc[3 * nqp + q]; sg[8] = mc[4 * nqp + q];
        sg[5] = sg[7] = mc[5 * nqp + q];
        sg[2] = sg[6] = mc[6 * nqp + q];
        sg[1] = sg[3] = mc[7 * nqp + q];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int k = 0; k < 3; ++k)
                S[i * 3 + k] += G[i * 3 + 0] * sg[0 * 3 + k] + G[i * 3 + 1] * sg[1 * 3 + k] +
                                G[i * 3 + 2] * sg[2 * 3 + k];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            Pm[i * 3 + k] = S[i * 3 + 0] * Ji[k * 3 + 0] + S[i * 3 + 1] * Ji[k * 3 + 1] +
                            S[i * 3 + 2] * Ji[k * 3 + 2];
}

// modal coefficients (sum_a s_a(m) u_a) of a hex8 nodal 3-vector field, nodes in the reference's
// corner order; M[0..6] = xi, eta, zeta, xi eta, xi zeta, eta zeta, xi eta zeta (mode 1 unused)
__device__ __forceinline__ void hex8_modes(const float (&u)[8][3], float (&M)[7][3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float p0 = u[1][c] + u[0][c], m0 = u[1][c] - u[0][c];
        const float p1 = u[2][c] + u[3][c], m1 = u[2][c] - u[3][c];
        const float p2 = u[5][c] + u[4][c], m2 = u[5][c] - u[4][c];
        const float p3 = u[6][c] + u[7][c], m3 = u[6][c] - u[7][c];
        const float q0 = p1 + p0, q1 = p1 - p0, q2 = p3 + p2, q3 = p3 - p2;
        const float r0 = m1 + m0, r1 = m1 - m0, r2 = m3 + m2, r3 = m3 - m2;
        M[0][c] = r2 + r0;  // xi
        M[1][c] = q3 + q1;  // eta
        M[2][c] = q2 - q0;  // zeta
        M[3][c] = r3 + r1;  // xi eta
        M[4][c] = r2 - r0;  // xi zeta
        M[5][c] = q3 - q1;  // eta zeta
        M[6][c] = r3 - r1;  // xi eta zeta
    }
}

// reference gradient at (x, e, z): D[i][k] = d u_i / d xi_k (times 8)
__device__ __forceinline__ void hex8_grad(const float (&M)[7][3], float x, float e, float z,
                                          float* D) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        D[i * 3 + 0] = M[0][i] + e * M[3][i] + z * M[4][i] + (e * z) * M[6][i];
        D[i * 3 + 1] = M[1][i] + x * M[3][i] + z * M[5][i] + (x * z) * M[6][i];
        D[i * 3 + 2] = M[2][i] + x * M[4][i] + e * M[5][i] + (x * e) * M[6][i];
    }
}

template <int NPE, int MODEL>
__global__ void __launch_bounds__(kApply32Threads, (MODEL == MODEL_J2 || MODEL == MODEL_LE) ? 4 : 1)
k_apply32(int E, const int* __restrict__ conn,
                                                             const float* __restrict__ md,
                                                             const float* __restrict__ mc,
                                                             long long nqp, float Kb,
                                                             const float* __restrict__ v,
                                                             float* __restrict__ ye,
                                                             const int* __restrict__ done) {
    using T = Topo<NPE>;
    constexpr int NQ = T::NQ;
    if (done && *done) return;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    float d[NPE][3], vv[NPE][3], y[NPE][3];
    {
        const float4* m4 = reinterpret_cast<const float4*>(md + e * NPE * 3);
#pragma unroll
        for (int j = 0; j < NPE * 3 / 4; ++j) {
            const float4 t = m4[j];
            (&d[0][0])[4 * j + 0] = t.x;
            (&d[0][0])[4 * j + 1] = t.y;
            (&d[0][0])[4 * j + 2] = t.z;
            (&d[0][0])[4 * j + 3] = t.w;
        }
        const int4* c4 = reinterpret_cast<const int4*>(conn + e * NPE);
#pragma unroll
        for (int j = 0; j < NPE / 4; ++j) {
            const int4 t = c4[j];
            const int nd[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int k = 0; k < 3; ++k) vv[4 * j + b][k] = v[3ll * nd[b] + k];
        }
    }
    if constexpr (NPE == 8) {
        float Md[7][3], Mv[7][3], Y[7][3];
        hex8_modes(d, Md);
        hex8_modes(vv, Mv);
#pragma unroll
        for (int m = 0; m < 7; ++m) Y[m][0] = Y[m][1] = Y[m][2] = 0.0f;
        constexpr float g = 0.57735026918962576f;  // 1/sqrt(3): the 2-point Gauss abscissa
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            // point l has the signs of corner l (hexahedron_quadrature.cpp order)
            const float x = ((l == 1) || (l == 2) || (l == 5) || (l == 6)) ? g : -g;
            const float ee = ((l == 2) || (l == 3) || (l == 6) || (l == 7)) ? g : -g;
            const float z = (l >= 4) ? g : -g;
            float J[9], Gx[9], Pm[9];
            hex8_grad(Md, x, ee, z, J);
            hex8_grad(Mv, x, ee, z, Gx);
            point_flux<MODEL>(J, Gx, mc, nqp, e * 8 + l, 1.0f / 512.0f, Kb, Pm);
            const float ez = ee * z, xz = x * z, xe = x * ee;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float P0 = Pm[i * 3 + 0], P1 = Pm[i * 3 + 1], P2 = Pm[i * 3 + 2];
                Y[0][i] += P0;
                Y[1][i] += P1;
                Y[2][i] += P2;
                Y[3][i] += ee * P0 + x * P1;
                Y[4][i] += z * P0 + x * P2;
                Y[5][i] += z * P1 + ee * P2;
                Y[6][i] += ez * P0 + xz * P1 + xe * P2;
            }
        }
        // back to nodes: y_a = sum_m s_a(m) Y_m (transposed butterfly; mode 1 carries nothing)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float a0_1 = -Y[2][c], a1_1 = Y[2][c];           // 1 -/+ zeta
            const float a0_e = Y[1][c] - Y[5][c], a1_e = Y[1][c] + Y[5][c];
            const float a0_x = Y[0][c] - Y[4][c], a1_x = Y[0][c] + Y[4][c];
            const float a0_xe = Y[3][c] - Y[6][c], a1_xe = Y[3][c] + Y[6][c];
            // z = 0 corners 0..3, z = 1 corners 4..7
            const float b00_1 = a0_1 - a0_e, b01_1 = a0_1 + a0_e;   // (y=0 / y=1, z=0)
            const float b00_x = a0_x - a0_xe, b01_x = a0_x + a0_xe;
            const float b10_1 = a1_1 - a1_e, b11_1 = a1_1 + a1_e;   // (y=0 / y=1, z=1)
            const float b10_x = a1_x - a1_xe, b11_x = a1_x + a1_xe;
            y[0][c] = b00_1 - b00_x;  // (x0 y0 z0)
            y[1][c] = b00_1 + b00_x;  // (x1 y0 z0)
            y[2][c] = b01_1 + b01_x;  // (x1 y1 z0)
            y[3][c] = b01_1 - b01_x;  // (x0 y1 z0)
            y[4][c] = b10_1 - b10_x;  // (x0 y0 z1)
            y[5][c] = b10_1 + b10_x;  // (x1 y0 z1)
            y[6][c] = b11_1 + b11_x;  // (x1 y1 z1)
            y[7][c] = b11_1 - b11_x;  // (x0 y1 z1)
        }
    } else {
#pragma unroll
        for (int a = 0; a < NPE; ++a) y[a][0] = y[a][1] = y[a][2] = 0.0f;
#pragma unroll
        for (int l = 0; l < NQ; ++l) {
            float J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            float Gx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int a = 0; a < NPE; ++a)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float gk = dNf<NPE>((l * NPE + a) * 3 + k);
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        J[i * 3 + k] += d[a][i] * gk;
                        Gx[i * 3 + k] += vv[a][i] * gk;
                    }
                }
            float Pm[9];
            point_flux<MODEL>(J, Gx, mc, nqp, e * NQ + l, 1.0f / 6.0f, Kb, Pm);
#pragma unroll
            for (int a = 0; a < NPE; ++a) {
                const float g0 = dNf<NPE>((l * NPE + a) * 3 + 0), g1 = dNf<NPE>((l * NPE + a) * 3 + 1),
                            g2 = dNf<NPE>((l * NPE + a) * 3 + 2);
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    y[a][i] += Pm[i * 3 + 0] * g0 + Pm[i * 3 + 1] * g1 + Pm[i * 3 + 2] * g2;
            }
        }
    }
    // one plane per local node: threads of consecutive elements write consecutive entries
#pragma unroll
    for (int a = 0; a < NPE; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) ye[((long long)a * E + e) * 3 + i] = y[a][i];
}
