// tb_adjoint.cu -- reverse mode of the explicit MPM step (sm_100a).
//
// The reference has no adjoint: these kernels differentiate the forward step of
// this library by hand (bin -> P2G -> grid update -> G2P, with the FLIP/PIC
// blend, Neo-Hookean or fluid stress and slip walls). Backwards, one step is
//   1. G2P^T   per particle: F_bar <- (I + dt L)^T F_bar, L_bar = dt F_bar F^T,
//              and the window's v / vn sensitivities scattered to the grid;
//              x_bar gathers w_bar grad w + H grad_w_bar.
//   2. grid^T  per node: (v_bar, vn_bar) -> (m_bar, mv_bar, f_bar) through
//              vn = mv / m, v = vn + dt f / m (walled components carry nothing).
//   3. P2G^T   per particle: gathers m_bar, mv_bar, f_bar over the window into
//              x_bar, v_bar, sigma_bar and V_bar, then through sigma(F) and
//              V = V0 det F into F_bar and the Lame sensitivities.
// H is the Hessian of the kernel with respect to x_p (per-axis second
// derivatives of the quadratic B-spline or uGIMP). The forward values (weights,
// grid velocities) are read in the state type T; every adjoint quantity is FP64.
// Both particle passes keep the (BW+3)^D halo tile of the block they work on
// in shared memory, so the gathers stay on chip; the scatter of 1. uses global
// FP64 atomics. G2P^T runs one CTA per block, P2G^T one CTA per chunk of 512
// particles of the block-sorted permutation.
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

constexpr int ADJ_THREADS = 128;
// P2G backwards walks the block-sorted permutation in chunks of ADJ_CHUNK
// particles, one chunk per CTA at a time, loading the halo tile of each block
// the chunk touches: a crowded block is shared by several CTAs and a sparse
// scene still fills the GPU.
constexpr int ADJ_CHUNK = 512;

// Block origin (first tile node per axis) of 0-based block b.
template <int D, class T, int BW>
__device__ __forceinline__ void block_origin(const DMesh<D, T>& M, int b, int (&org)[3]) {
    org[0] = org[1] = org[2] = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        org[d] = (b % M.nb[d]) * BW - 1;
        b /= M.nb[d];
    }
}

// Linear mesh index of tile node t (false if outside the mesh).
template <int D, class T, int TS>
__device__ __forceinline__ bool tile_node(const DMesh<D, T>& M, const int (&org)[3], int t, long long& lin) {
    int node[3] = {0, 0, 0}, rem = t;
    bool inside = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        node[d] = org[d] + rem % TS;
        rem /= TS;
        inside = inside && node[d] >= 0 && node[d] < M.n[d];
    }
    lin = 0;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) lin = lin * M.n[d] + (inside ? node[d] : 0);
    return inside;
}

// Tile offsets of the particle's window; false (and an error bit) if the window
// leaves the block tile.
template <int D, int TS>
__device__ __forceinline__ bool window_in_tile(const AdjAxes<D>& ax, const int (&org)[3], int (&q0)[3], int* err) {
    bool ok = true;
    q0[0] = q0[1] = q0[2] = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        q0[d] = ax.lo[d] - org[d];
        ok = ok && q0[d] >= 0 && q0[d] + 2 < TS;
    }
    if (!ok) atomicOr(err, ERR_TILE_RANGE);
    return ok;
}

template <int D, int TS>
__device__ __forceinline__ int tile_slot(const int (&q0)[3], const int (&idx)[3]) {
    return (D == 3) ? (q0[0] + idx[0]) + TS * ((q0[1] + idx[1]) + TS * (q0[2] + idx[2]))
                    : (q0[0] + idx[0]) + TS * (q0[1] + idx[1]);
}

// G2P backwards, one CTA per non-empty block: v and v - vn of the block's halo
// tile in shared memory for the gathers; the v / vn sensitivities go straight to
// the global FP64 grid with fire-and-forget atomics (an FP64 shared tile, where
// all of a block's particles collide on a few hundred nodes, measured 3.7x
// slower on the sphere scene). One CTA per block, not per chunk: chunks of one
// crowded block on several SMs scatter to the same nodes at once (measured 1.5x
// slower on the sphere scene).
template <int D, class T, int BW>
__global__ void __launch_bounds__(ADJ_THREADS) adj_g2p_kernel(DMesh<D, T> M, GView<T> G, PView<T> P, Scalars<T> s,
                                                              AdjView A, GradGrid GB,
                                                              const int* __restrict__ totals,
                                                              const int* __restrict__ blocklist,
                                                              const int* __restrict__ offsets,
                                                              const int* __restrict__ perm, int* err) {
    constexpr int TS = BW + 3, TN = (D == 3) ? TS * TS * TS : TS * TS;
    __shared__ T tin[2 * D * TN];         // v_r at [r TN + t], (v - vn)_r at [(D + r) TN + t]
    const double dt = s.dt64, alpha = double(s.alpha);
    const int nactive = totals[0], tid = threadIdx.x;
    for (int bi = blockIdx.x; bi < nactive; bi += gridDim.x) {
      {
        const int b = blocklist[bi] - 1;
        const int s0 = offsets[b], s1 = offsets[b + 1];
        int org[3];
        block_origin<D, T, BW>(M, b, org);
        for (int t = tid; t < TN; t += ADJ_THREADS) {
            long long lin;
            const bool inside = tile_node<D, T, TS>(M, org, t, lin);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const T vi = inside ? G.v[d][lin] : T(0), vni = inside ? G.vn[d][lin] : T(0);
                tin[d * TN + t] = vi;
                tin[(D + d) * TN + t] = vi - vni;
            }
        }
        __syncthreads();
        for (int j = s0 + tid; j < s1; j += ADJ_THREADS) {
            const long long p = perm[j] - 1;
            T x[3] = {T(0), T(0), T(0)};
#pragma unroll
            for (int d = 0; d < D; ++d) x[d] = P.x[d][p];
            const T l = P.l ? P.l[p] : s.gimp_l;
            double F[3][3] = {}, Fb[3][3] = {};
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    F[r][c] = P.F[r + c * D][p];
                    Fb[r][c] = A.F[r + c * D][p];
                }
            double xb[3] = {0, 0, 0}, vbp[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < D; ++d) {
                xb[d] = A.x[d][p];
                vbp[d] = A.v[d][p];
            }
            AdjAxes<D> ax;
            int q0[3];
            const bool in = adj_axes<D, T>(M, s, x, l, ax, err) && window_in_tile<D, TS>(ax, org, q0, err);
            double L[3][3] = {};
            if (in) {
#pragma unroll
                for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const int idx[3] = {i, jj, k};
                            if (i >= ax.cnt[0] || jj >= ax.cnt[1] || (D == 3 && k >= ax.cnt[D - 1])) continue;
                            double w, g[3], H[3][3];
                            adj_node<D>(ax, idx, w, g, H);
                            const int t = tile_slot<D, TS>(q0, idx);
#pragma unroll
                            for (int r = 0; r < D; ++r) {
                                const double vi = double(tin[r * TN + t]);
#pragma unroll
                                for (int c = 0; c < D; ++c) L[r][c] += vi * g[c];
                            }
                        }
            }
            double Lb[3][3] = {}, Fbn[3][3] = {};
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    double s1v = 0.0, s2v = 0.0;
#pragma unroll
                    for (int k = 0; k < D; ++k) {
                        s1v += ((r == k ? 1.0 : 0.0) + dt * L[k][r]) * Fb[k][c];
                        s2v += Fb[r][k] * F[c][k];
                    }
                    Fbn[r][c] = s1v;
                    Lb[r][c] = dt * s2v;
                }
            double dvb[3] = {0, 0, 0}, vpb[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < D; ++d) {
                dvb[d] = alpha * vbp[d];
                vpb[d] = (1.0 - alpha) * vbp[d] + dt * xb[d];
            }
            if (in) {
                long long gbase = 0;
#pragma unroll
                for (int d = D - 1; d >= 0; --d) gbase = gbase * M.n[d] + ax.lo[d];
#pragma unroll
                for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const int idx[3] = {i, jj, k};
                            if (i >= ax.cnt[0] || jj >= ax.cnt[1] || (D == 3 && k >= ax.cnt[D - 1])) continue;
                            double w, g[3], H[3][3];
                            adj_node<D>(ax, idx, w, g, H);
                            const int t = tile_slot<D, TS>(q0, idx);
                            const long long I = gbase + i + (long long)M.n[0] * (jj + (D == 3 ? (long long)M.n[1] * k : 0));
                            double gb[3] = {0, 0, 0}, wb = 0.0;
#pragma unroll
                            for (int r = 0; r < D; ++r) {
                                const double vi = double(tin[r * TN + t]), dvi = double(tin[(D + r) * TN + t]);
                                double lg = 0.0;
#pragma unroll
                                for (int c = 0; c < D; ++c) {
                                    lg += Lb[r][c] * g[c];
                                    gb[c] += Lb[r][c] * vi;
                                }
                                atomicAdd(GB.vb[r] + I, w * (vpb[r] + dvb[r]) + lg);
                                atomicAdd(GB.vnb[r] + I, -w * dvb[r]);
                                wb += vpb[r] * vi + dvb[r] * dvi;
                            }
#pragma unroll
                            for (int bb = 0; bb < D; ++bb) {
                                double h = 0.0;
#pragma unroll
                                for (int c = 0; c < D; ++c) h += H[bb][c] * gb[c];
                                xb[bb] += wb * g[bb] + h;
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
        __syncthreads();
      }
    }
}

// Particles outside the mesh: their G2P keeps x and F and scales v by alpha.
template <int D, class T>
__global__ void __launch_bounds__(256) adj_outside_kernel(long long n, const int* __restrict__ blockids, double alpha,
                                                          AdjView A) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        if (blockids[p] == 0) {
#pragma unroll
            for (int d = 0; d < D; ++d) A.v[d][p] *= alpha;
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

// P2G backwards, one CTA per chunk of the permutation: the block's halo tile of
// (m_bar, mv_bar, f_bar) in shared memory, gathered per particle, then the
// constitutive adjoint in FP64.
template <int D, class T, int BW>
__global__ void __launch_bounds__(ADJ_THREADS) adj_p2g_kernel(DMesh<D, T> M, PView<T> P, Scalars<T> s, AdjView A,
                                                              GradGrid GB, const int* __restrict__ totals,
                                                              const int* __restrict__ blockids,
                                                              const int* __restrict__ offsets,
                                                              const int* __restrict__ perm, int* err) {
    constexpr int TS = BW + 3, TN = (D == 3) ? TS * TS * TS : TS * TS;
    constexpr int NC = 1 + 2 * D;
    __shared__ double tg[NC * TN];  // m_bar at [t], mv_bar_d at [(1 + d) TN + t], f_bar_d at [(1 + D + d) TN + t]
    const int nassigned = totals[1], tid = threadIdx.x;
    const int nchunks = (nassigned + ADJ_CHUNK - 1) / ADJ_CHUNK;
    for (int ci = blockIdx.x; ci < nchunks; ci += gridDim.x) {
      const int c1 = min((ci + 1) * ADJ_CHUNK, nassigned);
      for (int c0 = ci * ADJ_CHUNK; c0 < c1;) {
        // the block of the chunk's next particle, and the part of the chunk in it
        const int b = blockids[perm[c0] - 1] - 1;
        const int s0 = c0, s1 = min(offsets[b + 1], c1);
        int org[3];
        block_origin<D, T, BW>(M, b, org);
        for (int t = tid; t < TN; t += ADJ_THREADS) {
            long long lin;
            const bool inside = tile_node<D, T, TS>(M, org, t, lin);
            tg[t] = inside ? GB.mb[lin] : 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                tg[(1 + d) * TN + t] = inside ? GB.pb[d][lin] : 0.0;
                tg[(1 + D + d) * TN + t] = inside ? GB.fb[d][lin] : 0.0;
            }
        }
        __syncthreads();
        for (int j = s0 + tid; j < s1; j += ADJ_THREADS) {
            const long long p = perm[j] - 1;
            T x[3] = {T(0), T(0), T(0)};
#pragma unroll
            for (int d = 0; d < D; ++d) x[d] = P.x[d][p];
            const T l = P.l ? P.l[p] : s.gimp_l;
            double xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0}, sb[3][3] = {}, Vb = 0.0;
            AdjAxes<D> ax;
            int q0[3];
            if (adj_axes<D, T>(M, s, x, l, ax, err) && window_in_tile<D, TS>(ax, org, q0, err)) {
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
                    for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const int idx[3] = {i, jj, k};
                            if (i >= ax.cnt[0] || jj >= ax.cnt[1] || (D == 3 && k >= ax.cnt[D - 1])) continue;
                            double w, g[3], H[3][3];
                            adj_node<D>(ax, idx, w, g, H);
                            const int t = tile_slot<D, TS>(q0, idx);
                            double wb = mp * tg[t];
                            double gb[3] = {0, 0, 0}, fbv[3] = {0, 0, 0};
#pragma unroll
                            for (int d = 0; d < D; ++d) {
                                const double pbd = tg[(1 + d) * TN + t];
                                fbv[d] = tg[(1 + D + d) * TN + t];
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
                            for (int bb = 0; bb < D; ++bb) {
                                double h = 0.0;
#pragma unroll
                                for (int c = 0; c < D; ++c) h += H[bb][c] * gb[c];
                                xb[bb] += wb * g[bb] + h;
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
                        double bsum = 0.0;
#pragma unroll
                        for (int k = 0; k < D; ++k) bsum += F[r][k] * F[c][k];
                        const double bm = bsum - (r == c ? 1.0 : 0.0);
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
        __syncthreads();
        c0 = s1;
      }
    }
}

}  // namespace

template <int D, class T, int BW>
cudaError_t launch_adjoint(const DMesh<D, T>& M, const GView<T>& G, const PView<T>& P, const Scalars<T>& s,
                           const AdjView& A, const GradGrid& GB, const AdjPartition& part, const LaunchCfg& cfg) {
    cudaError_t e = cudaSuccess;
    for (int d = 0; d < D && e == cudaSuccess; ++d) {
        e = cudaMemsetAsync(GB.vb[d], 0, sizeof(double) * size_t(M.nnodes), cfg.stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(GB.vnb[d], 0, sizeof(double) * size_t(M.nnodes), cfg.stream);
    }
    if (e != cudaSuccess) return e;
    const int bgrid = std::max(1, std::min(M.nblocks, cfg.num_sms * 8));
    const int cgrid = int(std::max<long long>(1, std::min<long long>((P.n + ADJ_CHUNK - 1) / ADJ_CHUNK,
                                                                     (long long)cfg.num_sms * 8)));
    const int ngrid = int(std::max<long long>(1, std::min<long long>((M.nnodes + 255) / 256, (long long)cfg.num_sms * 8)));
    if (P.n > 0) {
        KernelScope ks(cfg, "adj_g2p");
        adj_g2p_kernel<D, T, BW><<<bgrid, ADJ_THREADS, 0, cfg.stream>>>(M, G, P, s, A, GB, part.totals, part.blocklist,
                                                                       part.offsets, part.perm, cfg.err);
        ++*cfg.launches;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (s.alpha != T(1)) {
            const int pgrid = int(std::max<long long>(1, std::min<long long>((P.n + 255) / 256, (long long)cfg.num_sms * 8)));
            KernelScope ks2(cfg, "adj_outside");
            adj_outside_kernel<D, T><<<pgrid, 256, 0, cfg.stream>>>(P.n, part.blockids, double(s.alpha), A);
            ++*cfg.launches;
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
    }
    {
        KernelScope ks(cfg, "adj_grid");
        adj_grid_kernel<D, T><<<ngrid, 256, 0, cfg.stream>>>(M, G, s, GB);
        ++*cfg.launches;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (P.n > 0) {
        KernelScope ks(cfg, "adj_p2g");
        adj_p2g_kernel<D, T, BW><<<cgrid, ADJ_THREADS, 0, cfg.stream>>>(M, P, s, A, GB, part.totals, part.blockids,
                                                                       part.offsets, part.perm, cfg.err);
        ++*cfg.launches;
        e = cudaGetLastError();
    }
    return e;
}

#define TB_INST_ADJ(D, T, BW)                                                                                 \
    template cudaError_t launch_adjoint<D, T, BW>(const DMesh<D, T>&, const GView<T>&, const PView<T>&,       \
                                                  const Scalars<T>&, const AdjView&, const GradGrid&,         \
                                                  const AdjPartition&, const LaunchCfg&);
TB_INST_ADJ(3, double, 4)
TB_INST_ADJ(3, float, 4)
TB_INST_ADJ(2, double, 8)
TB_INST_ADJ(2, float, 8)
TB_INST_ADJ(2, double, 4)
TB_INST_ADJ(2, float, 4)

}  // namespace tb
