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
// In the FP64-position form (P.x64 set) the windows and in-window offsets come
// from the FP64 positions, as in the forward kernels of that form.
// Both particle passes keep the (BW+3)^D halo tile of the block they work on
// in shared memory, so the gathers stay on chip, and evaluate their sums over the
// window as separable moments (one axis at a time). The scatter of 1. is a
// separate pencil kernel with staged FP64 partials and one global atomic per
// node and block. The gathers run one CTA per chunk of 512 particles of the
// block-sorted permutation.
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

// Position of particle p in FP64: the FP64-position form's own array, else the
// state type's value.
template <int D, class T>
__device__ __forceinline__ void load_xd(const PView<T>& P, long long p, double (&xd)[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) xd[d] = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) xd[d] = P.x64[0] ? P.x64[d][p] : double(P.x[d][p]);
}

// Per-axis jets (value, first and second derivative in xi) of one particle's window.
template <int D>
struct AdjAxes {
    int lo[3], cnt[3];
    double val[3][3], der[3][3], d2[3][3];
    double hi;  // h_inv
};

template <int D, class T>
__device__ __forceinline__ bool adj_axes(const DMesh<D, T>& M, const Scalars<T>& s, const double* xd, bool x64,
                                         T l_abs, AdjAxes<D>& A, int* err) {
    Basis<D, T> B;
    if (x64) {
        if (!prepare_basis_x64<D, T>(M, s.basis, xd, l_abs, B, err)) return false;
    } else {
        const T x[3] = {T(xd[0]), T(xd[1]), T(xd[2])};
        if (!prepare_basis<D, T, false>(M, s.basis, x, l_abs, B, err)) return false;
    }
    const bool gimp = s.basis == TB_UGIMP;
    const double lnorm = gimp ? (x64 ? double(l_abs) / M.h64 : double(T(l_abs / M.h))) : 0.0;
    A.hi = x64 ? M.h_inv64 : double(M.h_inv);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        A.lo[d] = B.ax[d].lo;
        A.cnt[d] = B.ax[d].cnt;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            A.val[d][k] = double(B.ax[d].val[k]);
            A.der[d][k] = double(B.ax[d].der[k]);
            const double X = x64 ? __dadd_rn(M.xmin64[d], __dmul_rn(double(B.ax[d].lo + k), M.h64))
                                 : double(node_coord(M, d, B.ax[d].lo + k));
            const double xi = (xd[d] - X) * A.hi;
            A.d2[d][k] = (k < B.ax[d].cnt) ? (gimp ? d2_ugimp(xi, lnorm) : d2_bspline_quadratic(xi)) : 0.0;
        }
    }
    return true;
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

// Per-axis jets of one particle with the mesh scale folded in:
// J[d][0][k] = N, J[d][1][k] = N' h_inv, J[d][2][k] = N'' h_inv^2 at window slot
// k (zero past a truncated window and for d >= D).
template <int D>
__device__ __forceinline__ void axis_jets(const AdjAxes<D>& A, double (&J)[3][3][3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            J[d][0][k] = d < D ? A.val[d < D ? d : 0][k] : 0.0;
            J[d][1][k] = d < D ? A.der[d < D ? d : 0][k] * A.hi : 0.0;
            J[d][2][k] = d < D ? A.d2[d < D ? d : 0][k] * A.hi * A.hi : 0.0;
        }
}

// Slot of d2w / dx_a dx_b in a moment vector (see window_moments).
__host__ __device__ constexpr int hidx(int a, int b) {
    return a == b ? 4 + a : (a + b == 1 ? 7 : (a + b == 2 ? 8 : 9));
}

// Moments of one tile field phi over a particle's window: m[0] = sum w phi,
// m[1 + a] = sum (dw/dx_a) phi and, with ORD 2, m[hidx(a, b)] = sum
// (d2w/dx_a dx_b) phi, summed over the 3^D window nodes. w is a product of axis
// kernels, so the sums are contracted one axis at a time (x, then y, then z):
// 3 multiply-adds per window row and derivative order in x, then a few per row
// and plane, instead of forming w, grad w and the Hessian at every node.
// `t0` is the tile index of window slot (0, 0, 0).
template <int D, int ORD, int TS, class TT>
__device__ __forceinline__ void window_moments(const TT* __restrict__ phi, int t0, const double (&J)[3][3][3],
                                               double (&m)[10]) {
#pragma unroll
    for (int q = 0; q < 10; ++q) m[q] = 0.0;
#pragma unroll
    for (int k = 0; k < (D == 3 ? 3 : 1); ++k) {
        double y00 = 0.0, y10 = 0.0, y01 = 0.0, y20 = 0.0, y02 = 0.0, y11 = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const TT* r = phi + t0 + TS * (j + TS * k);
            const double f0 = double(r[0]), f1 = double(r[1]), f2 = double(r[2]);
            const double x0 = J[0][0][0] * f0 + J[0][0][1] * f1 + J[0][0][2] * f2;
            const double x1 = J[0][1][0] * f0 + J[0][1][1] * f1 + J[0][1][2] * f2;
            y00 += J[1][0][j] * x0;
            y10 += J[1][0][j] * x1;
            y01 += J[1][1][j] * x0;
            if constexpr (ORD == 2) {
                const double x2 = J[0][2][0] * f0 + J[0][2][1] * f1 + J[0][2][2] * f2;
                y20 += J[1][0][j] * x2;
                y02 += J[1][2][j] * x0;
                y11 += J[1][1][j] * x1;
            }
        }
        if constexpr (D == 3) {
            const double z0 = J[2][0][k], z1 = J[2][1][k];
            m[0] += z0 * y00;
            m[1] += z0 * y10;
            m[2] += z0 * y01;
            m[3] += z1 * y00;
            if constexpr (ORD == 2) {
                const double z2 = J[2][2][k];
                m[hidx(0, 0)] += z0 * y20;
                m[hidx(1, 1)] += z0 * y02;
                m[hidx(2, 2)] += z2 * y00;
                m[hidx(0, 1)] += z0 * y11;
                m[hidx(0, 2)] += z1 * y10;
                m[hidx(1, 2)] += z1 * y01;
            }
        } else {
            m[0] = y00;
            m[1] = y10;
            m[2] = y01;
            if constexpr (ORD == 2) {
                m[hidx(0, 0)] = y20;
                m[hidx(1, 1)] = y02;
                m[hidx(0, 1)] = y11;
            }
        }
    }
}

// G2P backwards, gather half, one CTA per chunk of the permutation: v and
// v - vn of the block's halo tile in shared memory. Per particle it forms
// L = sum v (x) grad w and the position sensitivity from window moments, writes
// the particle sensitivities, and leaves the coefficients of its grid scatter
//   v_bar_i += w a + Lb grad w,  vn_bar_i += w b
// (a = v_bar_p (1 - alpha) + dt x_bar + alpha v_bar_p, b = -alpha v_bar_p,
// Lb = dt F_bar F^T) at its permutation slot for adj_scatter_kernel.
template <int D, class T, int BW>
__global__ void __launch_bounds__(ADJ_THREADS) adj_g2p_kernel(DMesh<D, T> M, GView<T> G, PView<T> P, Scalars<T> s,
                                                              AdjView A, double* __restrict__ coef,
                                                              const int* __restrict__ totals,
                                                              const int* __restrict__ blockids,
                                                              const int* __restrict__ offsets,
                                                              const int* __restrict__ perm, int* err) {
    constexpr int TS = BW + 3, TN = (D == 3) ? TS * TS * TS : TS * TS;
    __shared__ T tin[2 * D * TN];  // v_r at [r TN + t], (v - vn)_r at [(D + r) TN + t]
    const double dt = s.dt64, alpha = double(s.alpha);
    const long long n = P.n;
    const int nassigned = totals[1], tid = threadIdx.x;
    const int nchunks = (nassigned + ADJ_CHUNK - 1) / ADJ_CHUNK;
    for (int ci = blockIdx.x; ci < nchunks; ci += gridDim.x) {
      const int c1 = min((ci + 1) * ADJ_CHUNK, nassigned);
      for (int c0 = ci * ADJ_CHUNK; c0 < c1;) {
        const int b = blockids[perm[c0] - 1] - 1;
        const int s0 = c0, s1 = min(offsets[b + 1], c1);
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
        int pnext = s0 + tid < s1 ? perm[s0 + tid] : 1;
        for (int j = s0 + tid; j < s1; j += ADJ_THREADS) {
            const long long p = pnext - 1;
            if (j + ADJ_THREADS < s1) pnext = perm[j + ADJ_THREADS];
            double xd[3];
            load_xd<D, T>(P, p, xd);
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
            // Lb = dt F_bar F^T does not depend on L
            double Lb[3][3] = {};
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    double s2v = 0.0;
#pragma unroll
                    for (int k = 0; k < D; ++k) s2v += Fb[r][k] * F[c][k];
                    Lb[r][c] = dt * s2v;
                }
            double dvb[3] = {0, 0, 0}, vpb[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < D; ++d) {
                dvb[d] = alpha * vbp[d];
                vpb[d] = (1.0 - alpha) * vbp[d] + dt * xb[d];
            }
            AdjAxes<D> ax;
            int q0[3];
            const bool in = adj_axes<D, T>(M, s, xd, P.x64[0] != nullptr, l, ax, err) && window_in_tile<D, TS>(ax, org, q0, err);
            double L[3][3] = {};
            if (in) {
                double J[3][3][3];
                axis_jets<D>(ax, J);
                const int zero[3] = {0, 0, 0};
                const int t0 = tile_slot<D, TS>(q0, zero);
                // x_bar += sum_i (vpb . v_i + dvb . dv_i) grad w + H (Lb^T v_i)
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    double mo[10];
                    window_moments<D, 2, TS>(tin + r * TN, t0, J, mo);
#pragma unroll
                    for (int c = 0; c < D; ++c) L[r][c] = mo[1 + c];
#pragma unroll
                    for (int bb = 0; bb < D; ++bb) {
                        double h = 0.0;
#pragma unroll
                        for (int c = 0; c < D; ++c) h += Lb[r][c] * mo[hidx(bb, c)];
                        xb[bb] += vpb[r] * mo[1 + bb] + h;
                    }
                    window_moments<D, 1, TS>(tin + (D + r) * TN, t0, J, mo);
#pragma unroll
                    for (int bb = 0; bb < D; ++bb) xb[bb] += dvb[r] * mo[1 + bb];
                }
            }
            double Fbn[3][3] = {};
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    double s1v = 0.0;
#pragma unroll
                    for (int k = 0; k < D; ++k) s1v += ((r == k ? 1.0 : 0.0) + dt * L[k][r]) * Fb[k][c];
                    Fbn[r][c] = s1v;
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
            double* q = coef + j;
#pragma unroll
            for (int r = 0; r < D; ++r) {
                q[r * n] = in ? vpb[r] + dvb[r] : 0.0;
                q[(D + r) * n] = in ? -dvb[r] : 0.0;
#pragma unroll
                for (int c = 0; c < D; ++c) q[(2 * D + r * D + c) * n] = in ? Lb[r][c] : 0.0;
            }
        }
        __syncthreads();
        c0 = s1;
      }
    }
}

// G2P backwards, scatter half: v_bar_i += w a + Lb grad w and vn_bar_i += w b
// from the coefficients adj_g2p_kernel left per permutation slot. The forward
// P2G's pencil sweep, in FP64, with the accumulators kept in registers across
// the batches of a block: per batch of up to SC_NR particles of one block the
// records are counting-sorted by window start (group); the lane of window row
// (y, z) of pencil (gy, gz) keeps the row's TS x-nodes in registers and adds
// every particle of the pencil's groups to the 3 of them its window covers.
// When the CTA moves to another block, the lanes store their rows to a staging
// array and one thread per tile node sums the at most 3^(D-1) rows that reach
// it and adds them to the grid with one global FP64 atomic per non-zero value
// (no shared atomics). A CTA takes a contiguous range of the permutation, so
// all batches of a crowded block share one flush.
constexpr int SC_THREADS = 288;
constexpr int SC_NR = 768;  // 3 particles per thread in the record pass
// Record (doubles): [0..2] a [3..5] b [6..14] Lb (r 3 + c) [16..21] x jets
// (value, h_inv-scaled derivative per slot) [22..27] y jets [28..33] z jets.
// 34 doubles = 17 x 16 bytes.
constexpr int SC_RS = 34;

template <int D, int BW>
struct ScShape {
    static constexpr int TS = BW + 3;
    static constexpr int TN = (D == 3) ? TS * TS * TS : TS * TS;
    static constexpr int NC = 2 * D;
    static constexpr int G1 = BW + 1;
    static constexpr int NG = (D == 3) ? G1 * G1 * G1 : G1 * G1;
    static constexpr int NJK = (D == 3) ? 9 : 3;
    static constexpr int NSUB = 32 / NJK;
    static constexpr int NPENCIL = NG / G1;
    static constexpr int CSTR = NPENCIL * NJK * TS;
    static constexpr int NPART = NC * CSTR;
    // records and staging share one region (never live at once)
    static constexpr int NDBL = (SC_NR * SC_RS > NPART) ? SC_NR * SC_RS : NPART;
};

template <int D, class T, int BW>
__global__ void __launch_bounds__(SC_THREADS, 1) adj_scatter_kernel(DMesh<D, T> M, PView<T> P, Scalars<T> s,
                                                                     const double* __restrict__ coef, GradGrid GB,
                                                                     const int* __restrict__ totals,
                                                                     const int* __restrict__ blockids,
                                                                     const int* __restrict__ offsets,
                                                                     const int* __restrict__ perm, long long per_cta,
                                                                     int* err) {
    using SH = ScShape<D, BW>;
    constexpr int NT = SC_THREADS, NW = NT / 32;
    constexpr int TS = SH::TS, TN = SH::TN, NC = SH::NC, G1 = SH::G1, NG = SH::NG;
    constexpr int NJK = SH::NJK, NSUB = SH::NSUB, NPENCIL = SH::NPENCIL, CSTR = SH::CSTR;
    static_assert((NPENCIL + NSUB - 1) / NSUB <= NW, "one pencil per lane");
    static_assert(NT % 8 == 0 && SC_NR % 8 == 0, "passes in 8-particle chunks");
    constexpr int ITEMS = (SC_NR + NT - 1) / NT;
    extern __shared__ __align__(16) double sc_smem[];
    double* rec = sc_smem;   // batch records, at the thread's slot
    double* part = sc_smem;  // staged rows at a flush
    int* gcount = reinterpret_cast<int*>(sc_smem + SH::NDBL);
    int* gstart = gcount + NG;
    int* order = gstart + NG + 1;  // record of the q-th particle in group order

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int jk = lane % NJK, sub = lane / NJK;
    const int sj = jk % 3, sk = (D == 3) ? jk / 3 : 0;
    const int pc = warp * NSUB + sub;  // this lane's pencil (gy + G1 gz)
    const bool live = sub < NSUB && pc < NPENCIL;
    const long long n = P.n;
    const double hi = double(M.h_inv);
    const int nassigned = totals[1];
    for (int g = tid; g < NG; g += NT) gcount[g] = 0;
    double acc[TS][NC];
#pragma unroll
    for (int x = 0; x < TS; ++x)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[x][c] = 0.0;
    __syncthreads();

    const long long lo_r = min((long long)blockIdx.x * per_cta, (long long)nassigned);
    const int r0 = int(lo_r), r1 = int(min(lo_r + per_cta, (long long)nassigned));
    // c0: start of the current block's segment of [r0, r1), taken in passes
    // that each sample the whole segment (BlockPasses); pass: the current one
    int c0 = r0, pass = 0;
    int b = c0 < r1 ? blockids[perm[c0] - 1] - 1 : -1;
    while (c0 < r1) {
        int org[3];
        block_origin<D, T, BW>(M, b, org);
        const int c1 = min(offsets[b + 1], r1);
        const BlockPasses bp(c0, c1, SC_NR);
        const bool last = pass + 1 >= bp.count();
        const int q0 = bp.pos(pass, tid), qstep = bp.step(NT);
        // the next batch's block, loaded early (uniform over the CTA)
        const int nb_next = !last ? b : (c1 < r1 ? blockids[perm[c1] - 1] - 1 : -1);
        // ---- 1a. particles tid, tid + NT, ...: window start -> group and rank in
        //      the group; the record goes to the particle's own slot. Every
        //      global load of the batch is issued before the first use.
        int grp[ITEMS], rank[ITEMS];
        long long pid[ITEMS];
#pragma unroll
        for (int u = 0; u < ITEMS; ++u) {
            grp[u] = -1;
            rank[u] = 0;
            const int q = q0 + u * qstep;
            pid[u] = (tid + u * NT < SC_NR && q < c1) ? perm[q] - 1 : -1;
        }
        double px[ITEMS][3];
        T pl[ITEMS];
#pragma unroll
        for (int u = 0; u < ITEMS; ++u) {
            const long long p = pid[u] >= 0 ? pid[u] : 0;
            load_xd<D, T>(P, p, px[u]);
            pl[u] = (pid[u] >= 0 && P.l) ? P.l[p] : s.gimp_l;
        }
        // the coefficients go to the record slot at once (used only if the
        // window lands in the tile)
#pragma unroll
        for (int u = 0; u < ITEMS; ++u) {
            if (pid[u] < 0) continue;
            const int j = q0 + u * qstep;
            double* r = rec + (tid + u * NT) * SC_RS;
#pragma unroll
            for (int rr = 0; rr < D; ++rr) {
                r[rr] = coef[rr * n + j];
                r[3 + rr] = coef[(D + rr) * n + j];
#pragma unroll
                for (int c = 0; c < D; ++c) r[6 + 3 * rr + c] = coef[(2 * D + rr * D + c) * n + j];
            }
        }
#pragma unroll
        for (int u = 0; u < ITEMS; ++u) {
            if (pid[u] < 0) continue;
            const int slot = tid + u * NT;
            Basis<D, T> B;
            bool in;
            if (P.x64[0]) {
                in = prepare_basis_x64<D, T>(M, s.basis, px[u], pl[u], B, err);
            } else {
                const T x[3] = {T(px[u][0]), T(px[u][1]), T(px[u][2])};
                in = prepare_basis<D, T, false>(M, s.basis, x, pl[u], B, err);
            }
            if (in) {
                int gi = 0;
                bool ok = true;
#pragma unroll
                for (int d = D - 1; d >= 0; --d) {
                    const int q = B.ax[d].lo - org[d];
                    ok = ok && q >= 0 && q < G1;
                    gi = gi * G1 + q;
                }
                if (ok) {  // (a window outside the tile is reported by the gather kernel)
                    grp[u] = gi;
                    rank[u] = atomicAdd(&gcount[gi], 1);
                    double* r = rec + slot * SC_RS;
#pragma unroll
                    for (int d = 0; d < D; ++d)
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            r[16 + 6 * d + 2 * k] = double(B.ax[d].val[k]);
                            r[17 + 6 * d + 2 * k] = double(B.ax[d].der[k]) * hi;
                        }
                }
            }
        }
        __syncthreads();
        if (warp == 0) {
            int carry = 0;
            for (int g0 = 0; g0 < NG; g0 += 32) {
                const int g = g0 + lane;
                const int c = g < NG ? gcount[g] : 0;
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                if (g < NG) gstart[g] = carry + incl - c;
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) gstart[NG] = carry;
        }
        __syncthreads();
        // ---- 1b. group order
        for (int g = tid; g < NG; g += NT) gcount[g] = 0;
#pragma unroll
        for (int u = 0; u < ITEMS; ++u)
            if (grp[u] >= 0) order[gstart[grp[u]] + rank[u]] = tid + u * NT;
        __syncthreads();
        // ---- 2. the lane's pencil: groups in x order, 3 register nodes each
        if (live) {
#pragma unroll
            for (int gx = 0; gx < G1; ++gx) {
                const int qe = gstart[G1 * pc + gx + 1];
                for (int q = gstart[G1 * pc + gx]; q < qe; ++q) {
                    const double* r = rec + order[q] * SC_RS;
                    const double2 yj = *reinterpret_cast<const double2*>(r + 22 + 2 * sj);
                    double wyz, dyz, wdz = 0.0;
                    if constexpr (D == 3) {
                        const double2 zk = *reinterpret_cast<const double2*>(r + 28 + 2 * sk);
                        wyz = yj.x * zk.x;
                        dyz = yj.y * zk.x;
                        wdz = yj.x * zk.y;
                    } else {
                        wyz = yj.x;
                        dyz = yj.y;
                    }
                    // per component: w a + Lb grad w = wx (a wyz + Lb1 dyz + Lb2 wdz) + dx Lb0 wyz
                    double AQ[3], Pc[3], Bv[3];
#pragma unroll
                    for (int rr = 0; rr < D; ++rr) {
                        double q2 = r[6 + 3 * rr + 1] * dyz;
                        if constexpr (D == 3) q2 += r[6 + 3 * rr + 2] * wdz;
                        AQ[rr] = r[rr] * wyz + q2;
                        Pc[rr] = r[6 + 3 * rr] * wyz;
                        Bv[rr] = r[3 + rr] * wyz;
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const double2 xj = *reinterpret_cast<const double2*>(r + 16 + 2 * i);
#pragma unroll
                        for (int rr = 0; rr < D; ++rr) {
                            acc[gx + i][rr] += xj.x * AQ[rr] + xj.y * Pc[rr];
                            acc[gx + i][D + rr] += xj.x * Bv[rr];
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (last) {
            c0 = c1;
            pass = 0;
        } else {
            ++pass;
        }
        if (nb_next != b) {
            // ---- 3. flush the block: rows to the staging array, then per tile
            //      node the staged rows, one global atomic per non-zero value
            if (live) {
                const int pbase = (jk * NPENCIL + pc) * TS;
#pragma unroll
                for (int x = 0; x < TS; ++x)
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        part[pbase + x + c * CSTR] = acc[x][c];
                        acc[x][c] = 0.0;
                    }
            }
            __syncthreads();
            for (int t = tid; t < TN; t += NT) {
                int node[3] = {0, 0, 0}, tn[3] = {0, 0, 0}, rem = t;
                bool inside = true;
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    tn[d] = rem % TS;
                    rem /= TS;
                    node[d] = org[d] + tn[d];
                    inside = inside && node[d] >= 0 && node[d] < M.n[d];
                }
                if (!inside) continue;
                double val[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) val[c] = 0.0;
#pragma unroll
                for (int kk = 0; kk < (D == 3 ? 3 : 1); ++kk)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj) {
                        const int gy = tn[1] - jj, gz = (D == 3) ? tn[2] - kk : 0;
                        if (gy < 0 || gy >= G1 || gz < 0 || gz >= G1) continue;
                        const int idx = ((jj + 3 * kk) * NPENCIL + gy + G1 * gz) * TS + tn[0];
#pragma unroll
                        for (int c = 0; c < NC; ++c) val[c] += part[idx + c * CSTR];
                    }
                long long lin = 0;
#pragma unroll
                for (int d = D - 1; d >= 0; --d) lin = lin * M.n[d] + node[d];
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    if (val[r] != 0.0) atomicAdd(GB.vb[r] + lin, val[r]);
                    if (val[D + r] != 0.0) atomicAdd(GB.vnb[r] + lin, val[D + r]);
                }
            }
            __syncthreads();
        }
        b = nb_next;
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

// P2G backwards, gather half, one CTA per chunk of the permutation: the
// block's halo tile of (m_bar, mv_bar, f_bar) in shared memory, gathered per
// particle as window moments into x_bar and v_bar; sigma_bar (D^2) and V_bar go
// to the scratch at the particle's index for adj_material_kernel.
template <int D, class T, int BW>
__global__ void __launch_bounds__(ADJ_THREADS) adj_p2g_kernel(DMesh<D, T> M, PView<T> P, Scalars<T> s, AdjView A,
                                                              GradGrid GB, double* __restrict__ sbar,
                                                              const int* __restrict__ totals,
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
        int pnext = s0 + tid < s1 ? perm[s0 + tid] : 1;
        for (int j = s0 + tid; j < s1; j += ADJ_THREADS) {
            const long long p = pnext - 1;
            if (j + ADJ_THREADS < s1) pnext = perm[j + ADJ_THREADS];
            double xd[3];
            load_xd<D, T>(P, p, xd);
            const T l = P.l ? P.l[p] : s.gimp_l;
            double xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0}, sb[3][3] = {}, Vb = 0.0;
            AdjAxes<D> ax;
            int q0[3];
            if (adj_axes<D, T>(M, s, xd, P.x64[0] != nullptr, l, ax, err) && window_in_tile<D, TS>(ax, org, q0, err)) {
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
                // Window moments of each grid sensitivity field:
                //   x_bar += m_p sum (m_bar + v . mv_bar + g . f_bar) grad w
                //            - V_p H sigma f_bar,
                //   v_bar += m_p sum w mv_bar,  sigma_bar = -V_p sum f_bar (x) grad w,
                //   V_bar = -sum f_bar . sigma grad w.
                double J[3][3][3];
                axis_jets<D>(ax, J);
                const int zero[3] = {0, 0, 0};
                const int t0 = tile_slot<D, TS>(q0, zero);
                double mo[10];
                window_moments<D, 1, TS>(tg, t0, J, mo);
#pragma unroll
                for (int bb = 0; bb < D; ++bb) xb[bb] += mp * mo[1 + bb];
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    window_moments<D, 1, TS>(tg + (1 + d) * TN, t0, J, mo);
                    vb[d] += mp * mo[0];
#pragma unroll
                    for (int bb = 0; bb < D; ++bb) xb[bb] += mp * vp[d] * mo[1 + bb];
                }
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    window_moments<D, 2, TS>(tg + (1 + D + r) * TN, t0, J, mo);
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        sb[r][c] += -Vp * mo[1 + c];
                        Vb += -sig[r][c] * mo[1 + c];
                    }
#pragma unroll
                    for (int bb = 0; bb < D; ++bb) {
                        double h = 0.0;
#pragma unroll
                        for (int c = 0; c < D; ++c) h += sig[r][c] * mo[hidx(bb, c)];
                        xb[bb] += mp * grav[r] * mo[1 + bb] - Vp * h;
                    }
                }
            }
#pragma unroll
            for (int d = 0; d < D; ++d) {
                A.x[d][p] += xb[d];
                A.v[d][p] += vb[d];
            }
            const long long n = P.n;
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) sbar[(r * D + c) * n + p] = sb[r][c];
            sbar[D * D * n + p] = Vb;
        }
        __syncthreads();
        c0 = s1;
      }
    }
}

// sigma(F) and V = V0 det F backwards (FP64), one thread per particle in memory
// order (particles outside the mesh, block 0, have no P2G part): sigma_bar and
// V_bar from adj_p2g_kernel into F_bar and the Lame sensitivities.
template <int D, class T>
__global__ void __launch_bounds__(256) adj_material_kernel(PView<T> P, Scalars<T> s, AdjView A,
                                                           const double* __restrict__ sbar,
                                                           const int* __restrict__ blockids) {
    const long long n = P.n;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        if (blockids[p] == 0) continue;
        double sb[3][3] = {};
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) sb[r][c] = sbar[(r * D + c) * n + p];
        const double Vb = sbar[D * D * n + p];
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
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) A.F[r + c * D][p] += Fb[r][c] + Jb * C[r][c];
        if (A.mu) A.mu[p] += mub;
        if (A.lam) A.lam[p] += lamb;
    }
}

// ---------------------------------------------------------------------------
// General reverse step (WLS and KernelCorrection bases, the APIC transfer): the
// oracle's general reverse step on the device, one thread per particle. The
// weights N_i, grad N_i and their derivatives with respect to x_p come from the
// basis evaluated in Dual3 (value plus the three x_p derivatives), so no
// second derivative of a WLS or corrected kernel is written out by hand. The
// v / vn sensitivities of G2P backwards are scattered with FP64 global atomics
// (27 nodes x 2D per particle); P2G backwards gathers m_bar, mv_bar, f_bar over
// the window and leaves sigma_bar, V_bar for adj_material_kernel.
// The mesh in Dual3: the state type's spacing and origin, or the FP64 ones in
// the FP64-position form (whose forward windows come from them).
template <int D, class T>
__device__ __forceinline__ DMesh<D, Dual3> dual_mesh(const DMesh<D, T>& M, bool x64) {
    DMesh<D, Dual3> R;
    for (int d = 0; d < 3; ++d) {
        R.n[d] = M.n[d];
        R.nb[d] = M.nb[d];
        R.xmin[d] = Dual3(x64 ? M.xmin64[d] : double(M.xmin[d]));
        R.xmin64[d] = M.xmin64[d];
    }
    R.L = M.L;
    R.nblocks = M.nblocks;
    R.nnodes = M.nnodes;
    R.h = Dual3(x64 ? M.h64 : double(M.h));
    R.h_inv = Dual3(x64 ? M.h_inv64 : double(M.h_inv));
    R.h64 = M.h64;
    R.h_inv64 = M.h_inv64;
    return R;
}

// Basis of particle x in Dual3: dual seeds e_0 .. e_{D-1} on the position.
template <int D, class T>
__device__ __forceinline__ bool dual_basis(const DMesh<D, Dual3>& MD, const Scalars<T>& s, const double* x, T l,
                                           Basis<D, Dual3>& B, int* err) {
    Dual3 xd[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        xd[d] = Dual3(d < D ? x[d] : 0.0);
        if (d < D) xd[d].d[d] = 1.0;
    }
    return prepare_basis<D, Dual3, true>(MD, s.basis, xd, Dual3(double(l)), B, err);
}

// N, grad N (values and x_p derivatives) at window slot (i, j, k), r = X - x_p.
template <int D>
__device__ __forceinline__ void dual_node(const DMesh<D, Dual3>& MD, const Basis<D, Dual3>& B, int i, int j, int k,
                                          const Dual3* rel, Dual3& N, Dual3* G) {
    eval_node<D, Dual3>(MD, B, i, j, k, rel, N, G);
}

template <int D, class T>
__global__ void __launch_bounds__(128) adj_g2p_gen_kernel(DMesh<D, T> M, GView<T> G, PView<T> P, Scalars<T> s,
                                                          AdjView A, GradGrid GB, const int* __restrict__ blockids,
                                                          int* err) {
    const DMesh<D, Dual3> MD = dual_mesh<D, T>(M, P.x64[0] != nullptr);
    const bool apic = s.transfer == TB_TRANSFER_APIC;
    const double dt = s.dt64, alpha = double(s.alpha);
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P.n;
         p += (long long)gridDim.x * blockDim.x) {
        double x[3];
        load_xd<D, T>(P, p, x);
        const T l = P.l ? P.l[p] : s.gimp_l;
        Basis<D, Dual3> B;
        const bool in = blockids[p] != 0 && dual_basis<D, T>(MD, s, x, l, B, err);
        double F[3][3] = {}, Fb[3][3] = {}, L[3][3] = {};
        load_F<D, T>(P, p, F);
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) Fb[r][c] = A.F[r + c * D][p];
        auto node_of = [&](int i, int j, int k, long long& I, Dual3 (&rel)[3], bool& valid) {
            const int idx[3] = {i, j, k};
            I = 0;
            valid = true;
#pragma unroll
            for (int d = D - 1; d >= 0; --d) {
                valid = valid && idx[d] < B.ax[d].cnt;
                I = I * M.n[d] + min(B.ax[d].lo + idx[d], M.n[d] - 1);
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) rel[d] = Dual3(0.0);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                rel[d] = node_coord(MD, d, B.ax[d].lo + idx[d]) - Dual3(x[d]);
                rel[d].d[d] = -1.0;
            }
        };
        if (in) {
            for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
                for (int j = 0; j < 3; ++j)
                    for (int i = 0; i < 3; ++i) {
                        long long I;
                        Dual3 rel[3];
                        bool valid;
                        node_of(i, j, k, I, rel, valid);
                        if (!valid) continue;
                        Dual3 N, Gn[3];
                        dual_node<D>(MD, B, i, j, k, rel, N, Gn);
#pragma unroll
                        for (int r = 0; r < D; ++r)
#pragma unroll
                            for (int c = 0; c < D; ++c) L[r][c] += double(G.v[r][I]) * Gn[c].v;
                    }
        }
        double Lb[3][3] = {}, Fbn[3][3] = {};
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) {
                double s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    s1 += ((r == q ? 1.0 : 0.0) + dt * L[q][r]) * Fb[q][c];
                    s2 += Fb[r][q] * F[c][q];
                }
                Fbn[r][c] = s1;
                Lb[r][c] = dt * s2;
            }
        double xb[3] = {}, vbp[3] = {}, vpicb[3] = {}, dvb[3] = {}, Bb[3][3] = {};
#pragma unroll
        for (int d = 0; d < D; ++d) {
            xb[d] = A.x[d][p];
            vbp[d] = A.v[d][p];
            if (apic) {
                vpicb[d] = vbp[d] + dt * xb[d];
            } else {
                dvb[d] = alpha * vbp[d];
                vpicb[d] = (1.0 - alpha) * vbp[d] + dt * xb[d];
            }
        }
        if (apic) {
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) Bb[r][c] = A.B[r + c * D][p];
        }
        if (in) {
            for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
                for (int j = 0; j < 3; ++j)
                    for (int i = 0; i < 3; ++i) {
                        long long I;
                        Dual3 rel[3];
                        bool valid;
                        node_of(i, j, k, I, rel, valid);
                        if (!valid) continue;
                        Dual3 N, Gn[3];
                        dual_node<D>(MD, B, i, j, k, rel, N, Gn);
                        double vi[3] = {}, vni[3] = {};
#pragma unroll
                        for (int d = 0; d < D; ++d) {
                            vi[d] = double(G.v[d][I]);
                            vni[d] = double(G.vn[d][I]);
                        }
                        double Nb = 0.0, Gb[3] = {0.0, 0.0, 0.0};
#pragma unroll
                        for (int r = 0; r < D; ++r) {
                            double vb_r = N.v * (vpicb[r] + dvb[r]);
#pragma unroll
                            for (int c = 0; c < D; ++c) vb_r += Lb[r][c] * Gn[c].v;
                            Nb += vpicb[r] * vi[r] + dvb[r] * (vi[r] - vni[r]);
#pragma unroll
                            for (int c = 0; c < D; ++c) Gb[c] += Lb[r][c] * vi[r];
                            if (apic) {
                                double Br = 0.0;
#pragma unroll
                                for (int c = 0; c < D; ++c) {
                                    Br += Bb[r][c] * rel[c].v;
                                    xb[c] -= N.v * vi[r] * Bb[r][c];
                                }
                                vb_r += N.v * Br;
                                Nb += vi[r] * Br;
                            }
                            atomicAdd(GB.vb[r] + I, vb_r);
                            if (!apic) atomicAdd(GB.vnb[r] + I, -N.v * dvb[r]);
                        }
#pragma unroll
                        for (int b = 0; b < D; ++b) {
                            double h = 0.0;
#pragma unroll
                            for (int c = 0; c < D; ++c) h += Gb[c] * Gn[c].d[b];
                            xb[b] += Nb * N.d[b] + h;
                        }
                    }
        }
#pragma unroll
        for (int d = 0; d < D; ++d) {
            A.x[d][p] = xb[d];
            A.v[d][p] = apic ? 0.0 : alpha * vbp[d];
        }
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) {
                A.F[r + c * D][p] = Fbn[r][c];
                if (apic) A.B[r + c * D][p] = 0.0;
            }
    }
}

template <int D, class T>
__global__ void __launch_bounds__(128) adj_p2g_gen_kernel(DMesh<D, T> M, PView<T> P, Scalars<T> s, AdjView A,
                                                          GradGrid GB, double* __restrict__ sbar,
                                                          const int* __restrict__ blockids, int* err) {
    const DMesh<D, Dual3> MD = dual_mesh<D, T>(M, P.x64[0] != nullptr);
    const bool apic = s.transfer == TB_TRANSFER_APIC;
    const double dinv = 4.0 / (double(M.h) * double(M.h));
    const long long n = P.n;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        if (blockids[p] == 0) continue;
        double x[3];
        load_xd<D, T>(P, p, x);
        const T l = P.l ? P.l[p] : s.gimp_l;
        Basis<D, Dual3> B;
        if (!dual_basis<D, T>(MD, s, x, l, B, err)) continue;
        const double mp = P.m ? double(P.m[p]) : double(s.mass);
        const double Vp = double(P.V[p]);
        double vp[3] = {}, Bp[3][3] = {}, sg[3][3] = {};
#pragma unroll
        for (int d = 0; d < D; ++d) vp[d] = double(P.v[d][p]);
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) {
                sg[r][c] = double(P.sig[symidx<D>(r, c)][p]);
                if (apic) Bp[r][c] = double(P.B[r + c * D][p]);
            }
        double xb[3] = {}, vbs[3] = {}, sb[3][3] = {}, Vb = 0.0, Bbs[3][3] = {};
        for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i) {
                    const int idx[3] = {i, j, k};
                    long long I = 0;
                    bool valid = true;
#pragma unroll
                    for (int d = D - 1; d >= 0; --d) {
                        valid = valid && idx[d] < B.ax[d].cnt;
                        I = I * M.n[d] + min(B.ax[d].lo + idx[d], M.n[d] - 1);
                    }
                    if (!valid) continue;
                    Dual3 rel[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) rel[d] = Dual3(0.0);
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        rel[d] = node_coord(MD, d, B.ax[d].lo + idx[d]) - Dual3(x[d]);
                        rel[d].d[d] = -1.0;
                    }
                    Dual3 N, Gn[3];
                    dual_node<D>(MD, B, i, j, k, rel, N, Gn);
                    double u[3] = {};
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        u[d] = vp[d];
                        if (apic)
#pragma unroll
                            for (int c = 0; c < D; ++c) u[d] += Bp[d][c] * dinv * rel[c].v;
                    }
                    double Nb = mp * GB.mb[I], Gb[3] = {0.0, 0.0, 0.0};
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        const double p_b = GB.pb[d][I], f_b = GB.fb[d][I];
                        Nb += mp * (u[d] * p_b + double(s.g[d]) * f_b);
                        const double ub = mp * N.v * p_b;
                        vbs[d] += ub;
                        if (apic)
#pragma unroll
                            for (int c = 0; c < D; ++c) {
                                Bbs[d][c] += ub * dinv * rel[c].v;
                                xb[c] -= ub * Bp[d][c] * dinv;
                            }
                    }
#pragma unroll
                    for (int r = 0; r < D; ++r) {
                        const double f_b = GB.fb[r][I];
                        double sgg = 0.0;
#pragma unroll
                        for (int c = 0; c < D; ++c) {
                            sgg += sg[r][c] * Gn[c].v;
                            Gb[c] += -Vp * sg[r][c] * f_b;
                            sb[r][c] += -Vp * f_b * Gn[c].v;
                        }
                        Vb += -f_b * sgg;
                    }
#pragma unroll
                    for (int b = 0; b < D; ++b) {
                        double h = 0.0;
#pragma unroll
                        for (int c = 0; c < D; ++c) h += Gb[c] * Gn[c].d[b];
                        xb[b] += Nb * N.d[b] + h;
                    }
                }
#pragma unroll
        for (int d = 0; d < D; ++d) {
            A.x[d][p] += xb[d];
            A.v[d][p] += vbs[d];
        }
        if (apic) {
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) A.B[r + c * D][p] += Bbs[r][c];
        }
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) sbar[(r * D + c) * n + p] = sb[r][c];
        sbar[D * D * n + p] = Vb;
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
    const int cgrid = int(std::max<long long>(1, std::min<long long>((P.n + ADJ_CHUNK - 1) / ADJ_CHUNK,
                                                                     (long long)cfg.num_sms * 8)));
    const int ngrid = int(std::max<long long>(1, std::min<long long>((M.nnodes + 255) / 256, (long long)cfg.num_sms * 8)));
    if (P.n > 0) {
        {
            KernelScope ks(cfg, "adj_g2p");
            adj_g2p_kernel<D, T, BW><<<cgrid, ADJ_THREADS, 0, cfg.stream>>>(M, G, P, s, A, GB.coef, part.totals,
                                                                           part.blockids, part.offsets, part.perm,
                                                                           cfg.err);
            ++*cfg.launches;
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        {
            using SH = ScShape<D, BW>;
            auto kern = adj_scatter_kernel<D, T, BW>;
            const size_t smem = sizeof(double) * size_t(SH::NDBL) + sizeof(int) * size_t(SH::NG + SH::NG + 1 + SC_NR);
            if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))) != cudaSuccess)
                return e;
            int per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SC_THREADS, smem);
            const long long nbatch = (P.n + SC_NR - 1) / SC_NR;
            const int sgrid = int(std::max<long long>(1, std::min<long long>(nbatch, (long long)cfg.num_sms * std::max(per_sm, 1))));
            const long long per_cta = ((nbatch + sgrid - 1) / sgrid) * SC_NR;
            KernelScope ks(cfg, "adj_scatter");
            kern<<<sgrid, SC_THREADS, smem, cfg.stream>>>(M, P, s, GB.coef, GB, part.totals, part.blockids, part.offsets,
                                                          part.perm, per_cta, cfg.err);
            ++*cfg.launches;
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
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
        {
            KernelScope ks(cfg, "adj_p2g");
            adj_p2g_kernel<D, T, BW><<<cgrid, ADJ_THREADS, 0, cfg.stream>>>(M, P, s, A, GB, GB.coef, part.totals,
                                                                           part.blockids, part.offsets, part.perm,
                                                                           cfg.err);
            ++*cfg.launches;
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        const int pgrid = int(std::max<long long>(1, std::min<long long>((P.n + 255) / 256, (long long)cfg.num_sms * 8)));
        KernelScope ks(cfg, "adj_material");
        adj_material_kernel<D, T><<<pgrid, 256, 0, cfg.stream>>>(P, s, A, GB.coef, part.blockids);
        ++*cfg.launches;
        e = cudaGetLastError();
    }
    return e;
}

template <int D, class T>
cudaError_t launch_adjoint_general(const DMesh<D, T>& M, const GView<T>& G, const PView<T>& P, const Scalars<T>& s,
                                   const AdjView& A, const GradGrid& GB, const AdjPartition& part, const LaunchCfg& cfg) {
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
        adj_g2p_gen_kernel<D, T><<<pgrid, 128, 0, cfg.stream>>>(M, G, P, s, A, GB, part.blockids, cfg.err);
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
        {
            KernelScope ks(cfg, "adj_p2g");
            adj_p2g_gen_kernel<D, T><<<pgrid, 128, 0, cfg.stream>>>(M, P, s, A, GB, GB.coef, part.blockids, cfg.err);
            ++*cfg.launches;
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        const int mgrid = int(std::max<long long>(1, std::min<long long>((P.n + 255) / 256, (long long)cfg.num_sms * 8)));
        KernelScope ks(cfg, "adj_material");
        adj_material_kernel<D, T><<<mgrid, 256, 0, cfg.stream>>>(P, s, A, GB.coef, part.blockids);
        ++*cfg.launches;
        e = cudaGetLastError();
    }
    return e;
}

#define TB_INST_ADJ(D, T, BW)                                                                                 \
    template cudaError_t launch_adjoint<D, T, BW>(const DMesh<D, T>&, const GView<T>&, const PView<T>&,       \
                                                  const Scalars<T>&, const AdjView&, const GradGrid&,         \
                                                  const AdjPartition&, const LaunchCfg&);
template cudaError_t launch_adjoint_general<3, double>(const DMesh<3, double>&, const GView<double>&,
                                                      const PView<double>&, const Scalars<double>&, const AdjView&,
                                                      const GradGrid&, const AdjPartition&, const LaunchCfg&);
template cudaError_t launch_adjoint_general<3, float>(const DMesh<3, float>&, const GView<float>&,
                                                     const PView<float>&, const Scalars<float>&, const AdjView&,
                                                     const GradGrid&, const AdjPartition&, const LaunchCfg&);
template cudaError_t launch_adjoint_general<2, double>(const DMesh<2, double>&, const GView<double>&,
                                                      const PView<double>&, const Scalars<double>&, const AdjView&,
                                                      const GradGrid&, const AdjPartition&, const LaunchCfg&);
template cudaError_t launch_adjoint_general<2, float>(const DMesh<2, float>&, const GView<float>&,
                                                     const PView<float>&, const Scalars<float>&, const AdjView&,
                                                     const GradGrid&, const AdjPartition&, const LaunchCfg&);
TB_INST_ADJ(3, double, 4)
TB_INST_ADJ(3, float, 4)
TB_INST_ADJ(2, double, 8)
TB_INST_ADJ(2, float, 8)
TB_INST_ADJ(2, double, 4)
TB_INST_ADJ(2, float, 4)

}  // namespace tb
