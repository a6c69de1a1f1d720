// element_kernel.cuh -- the fused element kernel (included by elements.cu).
//
// A group of G lanes owns one element (hex8: 8 lanes, 4 elements per warp; tet4: 2 lanes).
//   phase 0  gather node coordinates (X, x = u + X) into shared memory;
//   phase 1  lane l runs quadrature point l in FP64 (deformation measures, det F check,
//            constitutive update, current gradient L = dN J^-1, tangent coefficients); the
//            internal force of every node is reduced over the group with shuffles (hex8: a
//            reduce-scatter, so lane l ends with node l's force);
//   phase 2  hex8 in FP64 (every model but the anisotropic microspheres): each warp forms the
//            64 blocks of its elements, one element at a time, as 8x8 node x node tiles with
//            FP64 mma.sync, stages them in shared memory and adds them to K with red.global.add,
//            consecutive lanes on consecutive entries of a block (in a colour-partitioned pass,
//            A.order, an entry gets at most one term per launch, so the sums run in colour
//            order);
//            otherwise: each lane accumulates its upper-triangular 3x3 blocks over the points in
//            Real precision, in passes of at most 3 blocks (fewer live registers), and adds them
//            (and their mirrored blocks) to K with red.global.add.
// Shared memory per element holds L (Real) for every point, the flow direction N (J2) or the
// anisotropic tangent s Da (Langevin and non-affine microsphere) and, for finite-strain models,
// g = s sigma L (FP64) used by the geometric stiffness.
#pragma once

template <int NPE, int MODEL, typename Real, int MODE>
__global__ void __launch_bounds__(64, (MODEL == MODEL_J2) ? 8 : (model_aniso(MODEL) ? 4 : 8))
    k_element(ElementArgs A) {
    using T = Topo<NPE>;
    constexpr int NQ = T::NQ, G = T::G, EPC = T::EPC, MAXB = T::MAXB;
    constexpr bool kFinite = (MODEL == MODEL_NH || MODEL == MODEL_MS || model_aniso(MODEL));
    constexpr bool kJ2 = (MODEL == MODEL_J2);
    constexpr bool kAniso = model_aniso(MODEL);
    constexpr bool kCon = (MODE & MODE_CONSTITUTIVE) != 0;
    constexpr bool kStiff = (MODE & MODE_STIFFNESS) != 0;
    constexpr bool kForce = (MODE & MODE_FORCE) != 0;
    constexpr bool kStore = (MODE & MODE_STORE) != 0;
    // L per element: one row of NPE * 3 values per point.  hex8 pads each row to 25 doubles and
    // the element to 200: the 32 lanes of a warp (4 elements x 8 points) then store a row entry
    // in 2 shared-memory wavefronts instead of 8 (and the phase-2 loads stay at 4).
    constexpr int QS = (NPE == 8) ? NPE * 3 + 1 : NPE * 3;
    constexpr int LS = (NPE == 8) ? NQ * QS : NQ * QS + 2;
    // N (J2, 6 per point; an odd element stride puts the two elements of a half-warp on
    // different banks) or s Da
    constexpr int NS = kJ2 ? NQ * 6 + 1 : (kAniso ? NQ * 21 + 2 : 1);
    constexpr int GS = kFinite ? NQ * NPE * 3 + 1 : 1;  // g = s sigma L
    constexpr int NG = (NPE + G - 1) / G;          // nodes per lane
    // hex8 FP64 blocks on the FP64 mma.sync path (the anisotropic microsphere tangent keeps the
    // per-lane block loop)
    constexpr bool kMmaBlocks = (NPE == 8) && (sizeof(Real) == 8) && !kAniso;

    // phases 0-1 only: node coordinates and the reference gradients (one padding node per
    // point: the 8 points' rows, 27 doubles apart, fall on distinct banks)
    using XT = double[EPC][NPE][3];
    using DNT = double[NQ][NPE + 1][3];
    // mma path, phase 2 only: one element's 64 blocks per warp, staged so that consecutive lanes
    // reduce consecutive entries of a block (72 contiguous bytes in K); one padding double per
    // 16 blocks so that the 16 lanes of a half-warp write distinct banks.  It overlays the
    // phase 0-1 arrays: a barrier separates the two uses.
    constexpr int KS = kMmaBlocks ? NPE * NPE * 9 + 4 : 1;
    using KT = double[kMmaBlocks ? 2 : 1][KS];
    constexpr size_t kP01 = 2 * sizeof(XT) + sizeof(DNT);
    constexpr size_t kRaw = kP01 > sizeof(KT) ? kP01 : sizeof(KT);
    __shared__ __align__(16) unsigned char sRaw[kRaw];
    XT& sX = *reinterpret_cast<XT*>(sRaw);
    XT& sx = *reinterpret_cast<XT*>(sRaw + sizeof(XT));
    DNT& sdN = *reinterpret_cast<DNT*>(sRaw + 2 * sizeof(XT));
    KT& sKe = *reinterpret_cast<KT*>(sRaw);
    __shared__ Real sL[EPC][LS];
    __shared__ Real sN[EPC][NS];
    __shared__ double sG[EPC][GS];
    __shared__ Real sC[EPC][NQ][4];
    __shared__ int sSl[kMmaBlocks ? 2 : 1][kMmaBlocks ? NPE * NPE : 1];  // the staged blocks' slots

    const int tid = threadIdx.x;
    const int le = tid / G;
    const int lane = tid % G;
    const long long e = element_at(A, (long long)blockIdx.x * EPC + le);
    const bool valid = element_enabled(A, e);

    if constexpr (NPE != 8) {  // hex8 forms its derivatives in registers (hex8_dN)
        for (int i = tid; i < NQ * NPE * 3; i += blockDim.x)
            sdN[i / (NPE * 3)][(i % (NPE * 3)) / 3][i % 3] = c_dN_tet4[i];
    }

    // phase 0
    int node[NG];
#pragma unroll
    for (int j = 0; j < NG; ++j) {
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
            }
        }
    }
    __syncthreads();

    // phase 1
    double fown[NG][3];
#pragma unroll
    for (int j = 0; j < NG; ++j) fown[j][0] = fown[j][1] = fown[j][2] = 0.0;
    {
        const int l = lane;
        [[maybe_unused]] const Hex8Point hp = hex8_point(l);
        const bool active = valid && l < NQ;
        QpOut o;
        o.lam = o.mu = o.b = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) o.sig[c] = o.N[c] = 0.0;
        double Ji[9], s = 0.0;
        if (active) {
            const long long q = e * NQ + l;
            // the J2 history is loaded first, so its loads overlap the geometry below
            double ep_q[6] = {0, 0, 0, 0, 0, 0}, ebar_q = 0.0;
            if constexpr (kJ2 && kCon) {
#pragma unroll
                for (int c = 0; c < 6; ++c) ep_q[c] = A.ep[c * (long long)A.nqp + q];
                ebar_q = A.epbar[q];
            }
            // one pass over the nodes: F0 = X dN and U = (x - X) dN, then the current
            // Jacobian F = x dN = F0 + U, H = U F0^-1 (= sum_a (x_a - X_a) (x) (dN_a F0^-1),
            // submesh.cpp:225-231); without the update only F
            double Fc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            double F0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            double U[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int a = 0; a < NPE; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const double xi = sx[le][a][i], Xi = sX[le][a][i], di = xi - Xi;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        double d;
                        if constexpr (NPE == 8)
                            d = hex8_dN(hp, a, k);
                        else
                            d = sdN[l][a][k];
                        if constexpr (kCon) {
                            F0[i * 3 + k] += Xi * d;
                            U[i * 3 + k] += di * d;
                        } else {
                            Fc[i * 3 + k] += xi * d;
                        }
                    }
                }
            if constexpr (kCon) {
#pragma unroll
                for (int i = 0; i < 9; ++i) Fc[i] = F0[i] + U[i];
            }
            // J^-1 and w det J of the current configuration (submesh.cpp:82-160)
            const double detJ = inv3_det(Fc, Ji);
            s = ((NPE == 8) ? c_w_hex8[l] : (1.0 / 6.0)) * detJ;
            if constexpr (kCon) {
                double F0i[9];
                const double det0 = inv3_det(F0, F0i);
                double Hm[9];
                matmul3(U, F0i, Hm);
                // F_def = F F0^-1 (submesh.cpp:233); the small-strain models need only its
                // determinant, det F / det F0
                double Fd[9];
                double detF;
                if constexpr (kFinite) {
                    matmul3(Fc, F0i, Fd);
                    detF = det3(Fd);
                } else {
                    detF = detJ / det0;
                }
                if (signbit(detF)) {
                    const unsigned long long key = ((unsigned long long)q << 32) |
                                                   (unsigned long long)__float_as_uint((float)detF);
                    atomicMin(&A.status->negdet_first, key);
                    atomicAdd(&A.status->negdet_count, 1u);
                    report_status(A, e, NB2_E_NEG_DETJ);
                }
                // per-element moduli (batched instances, parameter fields) replace the material's
                const ElementArgs Ae = element_moduli(A, e);
                if constexpr (MODEL == MODEL_LE) {
                    cm_linear_elastic(Ae, Hm, o);
                } else if constexpr (MODEL == MODEL_NH) {
                    cm_neo_hooke(Ae, Fd, detF, o);
                } else if constexpr (MODEL == MODEL_J2) {
                    if (!cm_j2(A, q, Hm, o, ep_q, ebar_q)) report_status(A, e, NB2_E_RETURN_MAP);
                } else if constexpr (MODEL == MODEL_MS) {
                    cm_microsphere(Ae, Ae.G, Fd, detF, o);
                } else if constexpr (MODEL == MODEL_ML) {
                    cm_langevin(Ae, Ae.G, Fd, detF, o);
                } else {
                    cm_nonaffine(Ae, Ae.G, Fd, detF, o);
                }
                bool bad = isnan(o.lam) || isnan(o.mu);
#pragma unroll
                for (int c = 0; c < 6; ++c) bad |= isnan(o.sig[c]);
                if (bad) report_status(A, e, NB2_E_NAN);
                if constexpr (kStore) {
                    const long long n = A.nqp;
#pragma unroll
                    for (int c = 0; c < 6; ++c) A.sig[c * n + q] = o.sig[c];
                    A.dpar[0 * n + q] = o.lam;
                    A.dpar[1 * n + q] = o.mu;
                    A.dpar[2 * n + q] = o.b;
                    if constexpr (kAniso) {
#pragma unroll
                        for (int c = 0; c < 21; ++c) A.dpar[(3 + c) * n + q] = o.Da[c];
                    } else {
#pragma unroll
                        for (int c = 0; c < 6; ++c) A.dpar[(3 + c) * n + q] = kJ2 ? o.N[c] : 0.0;
                    }
                    A.detF[q] = detF;
                }
            } else {
                const long long n = A.nqp;
#pragma unroll
                for (int c = 0; c < 6; ++c) o.sig[c] = A.sig[c * n + q];
                o.lam = A.dpar[0 * n + q];
                o.mu = A.dpar[1 * n + q];
                o.b = A.dpar[2 * n + q];
                if constexpr (kAniso) {
#pragma unroll
                    for (int c = 0; c < 21; ++c) o.Da[c] = A.dpar[(3 + c) * n + q];
                } else {
#pragma unroll
                    for (int c = 0; c < 6; ++c) o.N[c] = A.dpar[(3 + c) * n + q];
                }
            }
        }
        if constexpr (kStiff || kForce) {
            // per node a: L_a = J^-T dN_a (stored for the stiffness phase) and g_a = s sigma L_a
            auto node_terms = [&](int a, double (&gv)[3]) {
                double La[3] = {0.0, 0.0, 0.0};
                if (active) {
                    double dn[3];
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        if constexpr (NPE == 8)
                            dn[m] = hex8_dN(hp, a, m);
                        else
                            dn[m] = sdN[l][a][m];
                    }
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                        La[k] = dn[0] * Ji[0 * 3 + k] + dn[1] * Ji[1 * 3 + k] + dn[2] * Ji[2 * 3 + k];
                }
                // sigma symmetric: 11 22 33 23 13 12
                gv[0] = s * (o.sig[0] * La[0] + o.sig[5] * La[1] + o.sig[4] * La[2]);
                gv[1] = s * (o.sig[5] * La[0] + o.sig[1] * La[1] + o.sig[3] * La[2]);
                gv[2] = s * (o.sig[4] * La[0] + o.sig[3] * La[1] + o.sig[2] * La[2]);
                if (active) {
                    if constexpr (kStiff) {
#pragma unroll
                        for (int k = 0; k < 3; ++k) sL[le][l * QS + 3 * a + k] = (Real)La[k];
                    }
                    if constexpr (kFinite && kStiff) {
#pragma unroll
                        for (int k = 0; k < 3; ++k) sG[le][l * NPE * 3 + 3 * a + k] = gv[k];
                    }
                }
            };
            if constexpr (NPE == 8 && G == 8 && kForce) {
                // internal force: a reduce-scatter over the 8 points of the group.  Each xor
                // round sends the half of the partial sums that the partner keeps, so lane l
                // ends with node l's sum (21 FP64 shuffles instead of 72); the additions are the
                // same tree as a full butterfly per node (own partial + partner's partial)
                const bool b2 = (lane & 4) != 0, b1 = (lane & 2) != 0, b0 = (lane & 1) != 0;
                double k1[4][3];
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    double gl[3], gu[3];
                    node_terms(p, gl);
                    node_terms(p + 4, gu);
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const double recv = __shfl_xor_sync(0xffffffffu, b2 ? gl[c] : gu[c], 4);
                        k1[p][c] = (b2 ? gu[c] : gl[c]) + recv;
                    }
                }
                double k2[2][3];
#pragma unroll
                for (int p = 0; p < 2; ++p)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const double x = k1[p][c], y = k1[p + 2][c];
                        const double recv = __shfl_xor_sync(0xffffffffu, b1 ? x : y, 2);
                        k2[p][c] = (b1 ? y : x) + recv;
                    }
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const double x = k2[0][c], y = k2[1][c];
                    const double recv = __shfl_xor_sync(0xffffffffu, b0 ? x : y, 1);
                    fown[0][c] = (b0 ? y : x) + recv;
                }
            } else {
#pragma unroll
                for (int a = 0; a < NPE; ++a) {
                    double gv[3];
                    node_terms(a, gv);
                    double g0 = gv[0], g1 = gv[1], g2 = gv[2];
                    if constexpr (kForce) {
                        // sum over the group's points (inactive lanes contribute zero)
#pragma unroll
                        for (int off = G / 2; off > 0; off >>= 1) {
                            g0 += __shfl_xor_sync(0xffffffffu, g0, off);
                            g1 += __shfl_xor_sync(0xffffffffu, g1, off);
                            g2 += __shfl_xor_sync(0xffffffffu, g2, off);
                        }
                        if (a % G == lane) {
                            fown[a / G][0] = g0;
                            fown[a / G][1] = g1;
                            fown[a / G][2] = g2;
                        }
                    }
                }
            }
            if (active) {
                if constexpr (kJ2 && kStiff) {
#pragma unroll
                    for (int c = 0; c < 6; ++c) sN[le][l * 6 + c] = (Real)o.N[c];
                }
                if constexpr (kAniso && kStiff) {
#pragma unroll
                    for (int c = 0; c < 21; ++c) sN[le][l * 21 + c] = (Real)(s * o.Da[c]);
                }
                sC[le][l][0] = (Real)(s * o.lam);
                sC[le][l][1] = (Real)(s * o.mu);
                sC[le][l][2] = (Real)(s * o.b);
                sC[le][l][3] = (Real)0;
            }
        }
    }
    __syncthreads();

    if constexpr (kForce) {
        if (valid) {
#pragma unroll
            for (int j = 0; j < NG; ++j) {
                const int a = lane + j * G;
                if (a < NPE) {
                    atomicAdd(&A.fint[3ll * node[j] + 0], fown[j][0]);
                    atomicAdd(&A.fint[3ll * node[j] + 1], fown[j][1]);
                    atomicAdd(&A.fint[3ll * node[j] + 2], fown[j][2]);
                }
            }
        }
    }

    if constexpr (kStiff && kMmaBlocks) {
        // hex8 FP64: each warp forms the 64 blocks of its 4 elements, one element at a time,
        // as 8x8 (node x node) products over the 8 points with mma.sync m8n8k4 (FP64).  Lane
        // (g, t) = (lane / 4, lane % 4) supplies the A operand (node g, point t + 4s) and the B
        // operand (point t + 4s, node g) of k-step s from the same shared values, and receives
        // the blocks (g, 2t) and (g, 2t + 1):
        //   K^ik = sum_q (s lam' L_qi)(L_qk)^T + (s mu' L_qk)(L_qi)^T
        //          + [i == k] sum_q sum_m (s mu' L_qm + s (sigma L)_qm)(L_qm)^T
        //          + sum_q (s b (N L)_qi)(N L)_qk^T                      (plastic J2 points)
        // -- the block formula above, all 64 blocks of the element, so no mirrored scatter.
        const int lane32 = tid & 31, warp = tid >> 5;
        const int g = lane32 >> 2, t = lane32 & 3;
        double* Kp = reinterpret_cast<double*>(A.K64);
#pragma unroll 1
        for (int j = 0; j < 4; ++j) {
            const int le2 = warp * 4 + j;
            const long long e2 = element_at(A, (long long)blockIdx.x * EPC + le2);
            if (!element_enabled(A, e2)) continue;  // the same for all lanes of the warp
            const int* slot = A.slot + e2 * (NPE * NPE);
            const int sl0 = slot[lane32], sl1 = slot[32 + lane32];
            double Lq[2][3], cl[2], cm[2], cb[2];
#pragma unroll
            for (int st = 0; st < 2; ++st) {
                const int q = t + 4 * st;
#pragma unroll
                for (int k = 0; k < 3; ++k) Lq[st][k] = (double)sL[le2][q * QS + 3 * g + k];
                cl[st] = (double)sC[le2][q][0];
                cm[st] = (double)sC[le2][q][1];
                cb[st] = (double)sC[le2][q][2];
            }
            // K is symmetric (K_ba[k][i] = K_ab[i][k]): only the component tiles i <= k are
            // formed; the diagonal ones merge their two products, and the staging writes each
            // off-diagonal value into both of its places
            constexpr int kTile[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
            double acc[6][2];
#pragma unroll
            for (int c = 0; c < 6; ++c) acc[c][0] = acc[c][1] = 0.0;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int st = 0; st < 2; ++st)
                    dmma_8x8x4(acc[kTile[i][i]], (cl[st] + cm[st]) * Lq[st][i], Lq[st][i]);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = i + 1; k < 3; ++k)
#pragma unroll
                    for (int st = 0; st < 2; ++st) {
                        dmma_8x8x4(acc[kTile[i][k]], cl[st] * Lq[st][i], Lq[st][k]);
                        dmma_8x8x4(acc[kTile[i][k]], cm[st] * Lq[st][k], Lq[st][i]);
                    }
            double sd[2] = {0.0, 0.0};
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
                for (int st = 0; st < 2; ++st) {
                    double av = cm[st] * Lq[st][m];
                    if constexpr (kFinite) av += sG[le2][(t + 4 * st) * NPE * 3 + 3 * g + m];
                    dmma_8x8x4(sd, av, Lq[st][m]);
                }
            if constexpr (kJ2) {
                if (__any_sync(0xffffffffu, cb[0] != 0.0 || cb[1] != 0.0)) {
                    double V[2][3];
#pragma unroll
                    for (int st = 0; st < 2; ++st) {
                        const Real* Nq = &sN[le2][(t + 4 * st) * 6];
                        const double N0 = Nq[0], N1 = Nq[1], N2 = Nq[2], N3 = Nq[3], N4 = Nq[4],
                                     N5 = Nq[5];
                        V[st][0] = N0 * Lq[st][0] + N5 * Lq[st][1] + N4 * Lq[st][2];
                        V[st][1] = N5 * Lq[st][0] + N1 * Lq[st][1] + N3 * Lq[st][2];
                        V[st][2] = N4 * Lq[st][0] + N3 * Lq[st][1] + N2 * Lq[st][2];
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int k = i; k < 3; ++k)
#pragma unroll
                            for (int st = 0; st < 2; ++st)
                                dmma_8x8x4(acc[kTile[i][k]], cb[st] * V[st][i], V[st][k]);
                }
            }
            sSl[warp][lane32] = sl0;
            sSl[warp][32 + lane32] = sl1;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int b = 2 * t + c;
                const int blk = g * NPE + b, blkT = b * NPE + g;
                double* Kab = &sKe[warp][blk * 9 + (blk >> 4)];
                double* Kba = &sKe[warp][blkT * 9 + (blkT >> 4)];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    Kab[4 * i] = acc[kTile[i][i]][c] + sd[c];
#pragma unroll
                    for (int k = i + 1; k < 3; ++k) {
                        Kab[3 * i + k] = acc[kTile[i][k]][c];
                        Kba[3 * k + i] = acc[kTile[i][k]][c];
                    }
                }
            }
            __syncwarp();
#pragma unroll 6
            for (int it = 0; it < NPE * NPE * 9 / 32; ++it) {
                const int idx = it * 32 + lane32;
                const int blk = idx / 9;
                const long long sab = sSl[warp][blk];
                atomicAdd(&Kp[9 * sab + (idx - 9 * blk)], sKe[warp][idx + (blk >> 4)]);
            }
            __syncwarp();
        }
        return;
    }

    if (!valid) return;

    if constexpr (kStiff) {
        const int* seg = (NPE == 8) ? c_seg_hex8[lane] : c_seg_tet4[lane];
        const int r0 = seg[0], b0s = seg[1], n0 = seg[2], r1 = seg[3], b1s = seg[4], n1 = seg[5];
        const int nb = n0 + n1;
        const int* slot = A.slot + e * (NPE * NPE);
        Real* Kp;
        if constexpr (sizeof(Real) == 8)
            Kp = reinterpret_cast<Real*>(A.K64);
        else
            Kp = reinterpret_cast<Real*>(A.K32);
        constexpr int PASS = 3;
#pragma unroll
        for (int jb = 0; jb < MAXB; jb += PASS) {
            if (jb >= nb) break;
            Real acc[PASS][9];
#pragma unroll
            for (int j = 0; j < PASS; ++j)
#pragma unroll
                for (int i = 0; i < 9; ++i) acc[j][i] = (Real)0;
            for (int l = 0; l < NQ; ++l) {
                const Real* Ll = &sL[le][l * QS];
                const Real cl = sC[le][l][0], cm = sC[le][l][1], cb = sC[le][l][2];
                Real Nq[6];
                if constexpr (kJ2) {
#pragma unroll
                    for (int c = 0; c < 6; ++c) Nq[c] = sN[le][l * 6 + c];
                }
                Real Lr0[3], Lr1[3], vr0[3], vr1[3], gr0[3], gr1[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    Lr0[k] = Ll[3 * r0 + k];
                    Lr1[k] = Ll[3 * r1 + k];
                    if constexpr (kFinite) {
                        gr0[k] = (Real)sG[le][l * NPE * 3 + 3 * r0 + k];
                        gr1[k] = (Real)sG[le][l * NPE * 3 + 3 * r1 + k];
                    }
                }
                if constexpr (kJ2) {
                    vr0[0] = Nq[0] * Lr0[0] + Nq[5] * Lr0[1] + Nq[4] * Lr0[2];
                    vr0[1] = Nq[5] * Lr0[0] + Nq[1] * Lr0[1] + Nq[3] * Lr0[2];
                    vr0[2] = Nq[4] * Lr0[0] + Nq[3] * Lr0[1] + Nq[2] * Lr0[2];
                    vr1[0] = Nq[0] * Lr1[0] + Nq[5] * Lr1[1] + Nq[4] * Lr1[2];
                    vr1[1] = Nq[5] * Lr1[0] + Nq[1] * Lr1[1] + Nq[3] * Lr1[2];
                    vr1[2] = Nq[4] * Lr1[0] + Nq[3] * Lr1[1] + Nq[2] * Lr1[2];
                }
#pragma unroll
                for (int jj = 0; jj < PASS; ++jj) {
                    const int j = jb + jj;
                    if (j < nb) {
                        const bool in0 = j < n0;
                        const int b = in0 ? b0s + j : b1s + (j - n0);
                        Real La[3], Lb[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            La[k] = in0 ? Lr0[k] : Lr1[k];
                            Lb[k] = Ll[3 * b + k];
                        }
                        const Real d = La[0] * Lb[0] + La[1] * Lb[1] + La[2] * Lb[2];
                        Real diag = cm * d;
                        if constexpr (kFinite) {
                            diag += (in0 ? gr0[0] : gr1[0]) * Lb[0] +
                                    (in0 ? gr0[1] : gr1[1]) * Lb[1] +
                                    (in0 ? gr0[2] : gr1[2]) * Lb[2];
                        }
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                Real v = cl * La[i] * Lb[k] + cm * La[k] * Lb[i];
                                if (i == k) v += diag;
                                acc[jj][3 * i + k] += v;
                            }
                        if constexpr (kAniso) aniso_block(&sN[le][l * 21], La, Lb, acc[jj]);
                        if constexpr (kJ2) {
                            if (cb != (Real)0) {
                                Real va[3], vb[3];
#pragma unroll
                                for (int k = 0; k < 3; ++k) va[k] = in0 ? vr0[k] : vr1[k];
                                vb[0] = Nq[0] * Lb[0] + Nq[5] * Lb[1] + Nq[4] * Lb[2];
                                vb[1] = Nq[5] * Lb[0] + Nq[1] * Lb[1] + Nq[3] * Lb[2];
                                vb[2] = Nq[4] * Lb[0] + Nq[3] * Lb[1] + Nq[2] * Lb[2];
#pragma unroll
                                for (int i = 0; i < 3; ++i)
#pragma unroll
                                    for (int k = 0; k < 3; ++k)
                                        acc[jj][3 * i + k] += cb * va[i] * vb[k];
                            }
                        }
                    }
                }
            }
            // scatter this pass: the block and (off the diagonal) its transpose
#pragma unroll
            for (int jj = 0; jj < PASS; ++jj) {
                const int j = jb + jj;
                if (j < nb) {
                    const bool in0 = j < n0;
                    const int a = in0 ? r0 : r1;
                    const int b = in0 ? b0s + j : b1s + (j - n0);
                    const long long sab = slot[a * NPE + b];
#pragma unroll
                    for (int i = 0; i < 9; ++i) atomicAdd(&Kp[9 * sab + i], acc[jj][i]);
                    if (a != b) {
                        const long long sba = slot[b * NPE + a];
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int k = 0; k < 3; ++k)
                                atomicAdd(&Kp[9 * sba + 3 * k + i], acc[jj][3 * i + k]);
                    }
                }
            }
        }
    }
}
