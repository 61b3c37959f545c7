// tb_adjoint.cu -- reverse mode of the explicit MPM step (sm_100a).
//
// The reference has no adjoint: these kernels differentiate the forward step of
// this library by hand (bin -> P2G -> grid update -> G2P, with the FLIP/PIC
// blend, Neo-Hookean or fluid stress and slip walls). Backwards, one step is
//   1. G2P^T   per particle: F_bar <- (I + dt L)^T F_bar, L_bar = dt F_bar F^T,
//              and the window's v / vn sensitivities scattered to the grid
//              (FP64 atomics); x_bar gathers w_bar grad w + H grad_w_bar.
//   2. grid^T  per node: (v_bar, vn_bar) -> (m_bar, mv_bar, f_bar) through
//              vn = mv / m, v = vn + dt f / m (walled components carry nothing).
//   3. P2G^T   per particle: gathers m_bar, mv_bar, f_bar over the window into
//              x_bar, v_bar, sigma_bar and V_bar, then through sigma(F) and
//              V = V0 det F into F_bar and the Lame sensitivities.
// H is the Hessian of the kernel with respect to x_p (per-axis second
// derivatives of the quadratic B-spline or uGIMP). The forward values (weights,
// grid velocities) are read in the state type T; every adjoint quantity is FP64.
#include "tb_launch.cuh"

namespace tb {

namespace {

__device__ __forceinline__ double d2_bspline_quadratic(double xi) {
    const double a = fabs(xi);
    return a < 0.5 ? -2.0 : (a < 1.5 ? 1.0 : 0.0);
}

__device__ __forceinline__ double d2_ugimp(double xi, double l) {
    const double a = fabs(xi);
    if (a < 0.5 * l) return -2.0 / l;
    if (a < 1.0 - 0.5 * l) return 0.0;
    if (a < 1.0 + 0.5 * l) return 1.0 / l;
    return 0.0;
}

// Per-axis jets (value, first and second derivative in xi) of one particle's window.
template <int D>
struct AdjAxes {
    int lo[3], cnt[3];
    double val[3][3], der[3][3], d2[3][3];
    double hi;  // h_inv
};

template <int D, class T>
__device__ __forceinline__ bool adj_axes(const DMesh<D, T>& M, const Scalars<T>& s, const T* x, T l_abs,
                                         AdjAxes<D>& A, int* err) {
    Basis<D, T> B;
    if (!prepare_basis<D, T, false>(M, s.basis, x, l_abs, B, err)) return false;
    const bool gimp = s.basis == TB_UGIMP;
    const double lnorm = gimp ? double(T(l_abs / M.h)) : 0.0;
    A.hi = double(M.h_inv);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        A.lo[d] = B.ax[d].lo;
        A.cnt[d] = B.ax[d].cnt;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            A.val[d][k] = double(B.ax[d].val[k]);
            A.der[d][k] = double(B.ax[d].der[k]);
            double xi = (double(x[d]) - double(node_coord(M, d, B.ax[d].lo + k))) * A.hi;
            A.d2[d][k] = (k < B.ax[d].cnt) ? (gimp ? d2_ugimp(xi, lnorm) : d2_bspline_quadratic(xi)) : 0.0;
        }
    }
    return true;
}

// w, grad w and the Hessian of w (with respect to x_p) at window slot idx.
template <int D>
__device__ __forceinline__ void adj_node(const AdjAxes<D>& A, const int (&idx)[3], double& w, double (&g)[3],
                                         double (&H)[3][3]) {
    w = 1.0;
#pragma unroll
    for (int d = 0; d < D; ++d) w *= A.val[d][idx[d]];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        double ga = A.der[a][idx[a]];
#pragma unroll
        for (int c = 0; c < D; ++c)
            if (c != a) ga *= A.val[c][idx[c]];
        g[a] = ga * A.hi;
#pragma unroll
        for (int b = 0; b < D; ++b) {
            double h = (a == b) ? A.d2[a][idx[a]] : A.der[a][idx[a]] * A.der[b][idx[b]];
#pragma unroll
            for (int c = 0; c < D; ++c)
                if (c != a && c != b) h *= A.val[c][idx[c]];
            H[a][b] = h * A.hi * A.hi;
        }
    }
}

template <int D, class T>
__device__ __forceinline__ long long adj_lin(const DMesh<D, T>& M, const AdjAxes<D>& A, const int (&idx)[3],
                                             bool& valid) {
    long long lin = 0;
    valid = true;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
        valid = valid && idx[d] < A.cnt[d];
        lin = lin * M.n[d] + min(A.lo[d] + idx[d], M.n[d] - 1);
    }
    return lin;
}

template <int D>
__device__ __forceinline__ double det_cof(const double (&F)[3][3], double (&C)[3][3]) {
    if constexpr (D == 3) {
        C[0][0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
        C[0][1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
        C[0][2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
        C[1][0] = F[0][2] * F[2][1] - F[0][1] * F[2][2];
        C[1][1] = F[0][0] * F[2][2] - F[0][2] * F[2][0];
        C[1][2] = F[0][1] * F[2][0] - F[0][0] * F[2][1];
        C[2][0] = F[0][1] * F[1][2] - F[0][2] * F[1][1];
        C[2][1] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
        C[2][2] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
        return F[0][0] * C[0][0] + F[0][1] * C[0][1] + F[0][2] * C[0][2];
    } else {
        C[0][0] = F[1][1];
        C[0][1] = -F[1][0];
        C[1][0] = -F[0][1];
        C[1][1] = F[0][0];
        return F[0][0] * F[1][1] - F[0][1] * F[1][0];
    }
}

template <int D, class T>
__global__ void __launch_bounds__(128) adj_g2p_kernel(DMesh<D, T> M, GView<T> G, PView<T> P, Scalars<T> s,
                                                      AdjView A, GradGrid GB, int* err) {
    const double dt = s.dt64, alpha = double(s.alpha);
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P.n;
         p += (long long)gridDim.x * blockDim.x) {
        T x[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int d = 0; d < D; ++d) x[d] = P.x[d][p];
        const T l = P.l ? P.l[p] : s.gimp_l;
        AdjAxes<D> ax;
        const bool in = adj_axes<D, T>(M, s, x, l, ax, err);
        double L[3][3] = {};
        if (in) {
#pragma unroll
            for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const int idx[3] = {i, j, k};
                        bool valid;
                        const long long I = adj_lin<D, T>(M, ax, idx, valid);
                        if (!valid) continue;
                        double w, g[3], H[3][3];
                        adj_node<D>(ax, idx, w, g, H);
#pragma unroll
                        for (int r = 0; r < D; ++r) {
                            const double vi = double(G.v[r][I]);
#pragma unroll
                            for (int c = 0; c < D; ++c) L[r][c] += vi * g[c];
                        }
                    }
        }
        double F[3][3] = {}, Fb[3][3] = {}, Lb[3][3] = {}, Fbn[3][3] = {};
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) {
                F[r][c] = P.F[r + c * D][p];
                Fb[r][c] = A.F[r + c * D][p];
            }
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) {
                double s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    s1 += ((r == k ? 1.0 : 0.0) + dt * L[k][r]) * Fb[k][c];
                    s2 += Fb[r][k] * F[c][k];
                }
                Fbn[r][c] = s1;
                Lb[r][c] = dt * s2;
            }
        double xb[3] = {0, 0, 0}, vbp[3] = {0, 0, 0}, dvb[3] = {0, 0, 0}, vpb[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < D; ++d) {
            xb[d] = A.x[d][p];
            vbp[d] = A.v[d][p];
            dvb[d] = alpha * vbp[d];
            vpb[d] = (1.0 - alpha) * vbp[d] + dt * xb[d];
        }
        if (in) {
#pragma unroll
            for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const int idx[3] = {i, j, k};
                        bool valid;
                        const long long I = adj_lin<D, T>(M, ax, idx, valid);
                        if (!valid) continue;
                        double w, g[3], H[3][3];
                        adj_node<D>(ax, idx, w, g, H);
                        double gb[3] = {0, 0, 0}, wb = 0.0;
#pragma unroll
                        for (int r = 0; r < D; ++r) {
                            const double vi = double(G.v[r][I]), vni = double(G.vn[r][I]);
                            double lg = 0.0;
#pragma unroll
                            for (int c = 0; c < D; ++c) {
                                lg += Lb[r][c] * g[c];
                                gb[c] += Lb[r][c] * vi;
                            }
                            atomicAdd(GB.vb[r] + I, w * (vpb[r] + dvb[r]) + lg);
                            atomicAdd(GB.vnb[r] + I, -w * dvb[r]);
                            wb += vpb[r] * vi + dvb[r] * (vi - vni);
                        }
#pragma unroll
                        for (int b = 0; b < D; ++b) {
                            double h = 0.0;
#pragma unroll
                            for (int c = 0; c < D; ++c) h += H[b][c] * gb[c];
                            xb[b] += wb * g[b] + h;
                        }
                    }
        }
#pragma unroll
        for (int d = 0; d < D; ++d) {
            A.x[d][p] = xb[d];
            A.v[d][p] = alpha * vbp[d];
        }
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) A.F[r + c * D][p] = Fbn[r][c];
    }
}

template <int D, class T>
__global__ void __launch_bounds__(256) adj_grid_kernel(DMesh<D, T> M, GView<T> G, Scalars<T> s, GradGrid GB) {
    const double dt = s.dt64;
    for (long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x; I < M.nnodes;
         I += (long long)gridDim.x * blockDim.x) {
        const double m = double(G.m[I]);
        int idx[3] = {0, 0, 0};
        long long r = I;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            idx[d] = int(r % M.n[d]);
            r /= M.n[d];
        }
        double acc = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            double v_b = GB.vb[d][I], vn_b = GB.vnb[d][I];
            const bool lo = (s.wall_mask >> (2 * d)) & 1, hi = (s.wall_mask >> (2 * d + 1)) & 1;
            if ((lo && idx[d] < s.wall_layers) || (hi && idx[d] >= M.n[d] - s.wall_layers)) v_b = vn_b = 0.0;
            double fb = 0.0, pb = 0.0;
            if (m != 0.0) {
                const double vt = vn_b + v_b;
                fb = dt * v_b / m;
                pb = vt / m;
                acc += vt * double(G.mv[d][I]) + dt * v_b * double(G.f[d][I]);
            }
            GB.fb[d][I] = fb;
            GB.pb[d][I] = pb;
        }
        GB.mb[I] = (m != 0.0) ? -acc / (m * m) : 0.0;
    }
}

template <int D, class T>
__global__ void __launch_bounds__(128) adj_p2g_kernel(DMesh<D, T> M, PView<T> P, Scalars<T> s, AdjView A,
                                                      GradGrid GB, int* err) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P.n;
         p += (long long)gridDim.x * blockDim.x) {
        T x[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int d = 0; d < D; ++d) x[d] = P.x[d][p];
        const T l = P.l ? P.l[p] : s.gimp_l;
        double xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0}, sb[3][3] = {}, Vb = 0.0;
        AdjAxes<D> ax;
        if (adj_axes<D, T>(M, s, x, l, ax, err)) {
            const double mp = double(P.m ? P.m[p] : s.mass), Vp = double(P.V[p]);
            double vp[3] = {0, 0, 0}, grav[3] = {0, 0, 0}, sig[3][3] = {};
#pragma unroll
            for (int d = 0; d < D; ++d) {
                vp[d] = double(P.v[d][p]);
                grav[d] = double(s.g[d]);
            }
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) sig[r][c] = double(P.sig[symidx<D>(r, c)][p]);
#pragma unroll
            for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const int idx[3] = {i, j, k};
                        bool valid;
                        const long long I = adj_lin<D, T>(M, ax, idx, valid);
                        if (!valid) continue;
                        double w, g[3], H[3][3];
                        adj_node<D>(ax, idx, w, g, H);
                        double wb = mp * GB.mb[I];
                        double gb[3] = {0, 0, 0}, fbv[3] = {0, 0, 0};
#pragma unroll
                        for (int d = 0; d < D; ++d) {
                            const double pbd = GB.pb[d][I];
                            fbv[d] = GB.fb[d][I];
                            wb += mp * (vp[d] * pbd + grav[d] * fbv[d]);
                            vb[d] += mp * w * pbd;
                        }
#pragma unroll
                        for (int r = 0; r < D; ++r) {
                            double sg = 0.0;
#pragma unroll
                            for (int c = 0; c < D; ++c) {
                                sg += sig[r][c] * g[c];
                                gb[c] += -Vp * sig[r][c] * fbv[r];
                                sb[r][c] += -Vp * fbv[r] * g[c];
                            }
                            Vb += -fbv[r] * sg;
                        }
#pragma unroll
                        for (int b = 0; b < D; ++b) {
                            double h = 0.0;
#pragma unroll
                            for (int c = 0; c < D; ++c) h += H[b][c] * gb[c];
                            xb[b] += wb * g[b] + h;
                        }
                    }
        }
        // sigma(F) and V = V0 det F backwards (FP64)
        double F[3][3] = {}, C[3][3] = {};
        load_F<D, T>(P, p, F);
        const double J = det_cof<D>(F, C);
        const double mu = P.mu ? double(P.mu[p]) : s.mu;
        const double lam = P.lam ? double(P.lam[p]) : s.lam;
        const double V0 = P.V0 ? double(P.V0[p]) : s.V0_64;
        double Jb = V0 * Vb, mub = 0.0, lamb = 0.0;
        double Fb[3][3] = {};
        if (s.material == 1) {
            double tr = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) tr += sb[d][d];
            lamb = (J - 1.0) * tr;
            Jb += lam * tr;
        } else {
            const double lj = log(J), iJ = 1.0 / J;
            double st = 0.0, trt = 0.0;
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    double b = 0.0;
#pragma unroll
                    for (int k = 0; k < D; ++k) b += F[r][k] * F[c][k];
                    const double bm = b - (r == c ? 1.0 : 0.0);
                    st += sb[r][c] * (mu * bm + (r == c ? lam * lj : 0.0));
                    mub += sb[r][c] * iJ * bm;
                }
#pragma unroll
            for (int d = 0; d < D; ++d) trt += sb[d][d] * iJ;
            Jb += -st * iJ * iJ + lam * trt * iJ;
            lamb = lj * trt;
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    double a = 0.0;
#pragma unroll
                    for (int k = 0; k < D; ++k) a += (sb[r][k] + sb[k][r]) * F[k][c];
                    Fb[r][c] = mu * iJ * a;
                }
        }
#pragma unroll
        for (int d = 0; d < D; ++d) {
            A.x[d][p] += xb[d];
            A.v[d][p] += vb[d];
        }
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) A.F[r + c * D][p] += Fb[r][c] + Jb * C[r][c];
        if (A.mu) A.mu[p] += mub;
        if (A.lam) A.lam[p] += lamb;
    }
}

}  // namespace

template <int D, class T>
cudaError_t launch_adjoint(const DMesh<D, T>& M, const GView<T>& G, const PView<T>& P, const Scalars<T>& s,
                           const AdjView& A, const GradGrid& GB, const LaunchCfg& cfg) {
    cudaError_t e = cudaSuccess;
    for (int d = 0; d < D && e == cudaSuccess; ++d) {
        e = cudaMemsetAsync(GB.vb[d], 0, sizeof(double) * size_t(M.nnodes), cfg.stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(GB.vnb[d], 0, sizeof(double) * size_t(M.nnodes), cfg.stream);
    }
    if (e != cudaSuccess) return e;
    const int pgrid = int(std::max<long long>(1, std::min<long long>((P.n + 127) / 128, (long long)cfg.num_sms * 16)));
    const int ngrid = int(std::max<long long>(1, std::min<long long>((M.nnodes + 255) / 256, (long long)cfg.num_sms * 8)));
    if (P.n > 0) {
        KernelScope ks(cfg, "adj_g2p");
        adj_g2p_kernel<D, T><<<pgrid, 128, 0, cfg.stream>>>(M, G, P, s, A, GB, cfg.err);
        ++*cfg.launches;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    {
        KernelScope ks(cfg, "adj_grid");
        adj_grid_kernel<D, T><<<ngrid, 256, 0, cfg.stream>>>(M, G, s, GB);
        ++*cfg.launches;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (P.n > 0) {
        KernelScope ks(cfg, "adj_p2g");
        adj_p2g_kernel<D, T><<<pgrid, 128, 0, cfg.stream>>>(M, P, s, A, GB, cfg.err);
        ++*cfg.launches;
        e = cudaGetLastError();
    }
    return e;
}

#define TB_INST_ADJ(D, T)                                                                                   \
    template cudaError_t launch_adjoint<D, T>(const DMesh<D, T>&, const GView<T>&, const PView<T>&,         \
                                              const Scalars<T>&, const AdjView&, const GradGrid&, const LaunchCfg&);
TB_INST_ADJ(3, double)
TB_INST_ADJ(3, float)
TB_INST_ADJ(2, double)
TB_INST_ADJ(2, float)

}  // namespace tb
