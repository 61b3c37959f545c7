// tb_common.cuh -- device-side data views and basis math shared by the kernels
// of libtesserae_b200.so (sm_100a).
//
// Mesh, window and weight rules follow the reference:
//   findblock / windows    Tesserae.jl src/Mesh/cartesian.jl:146-285
//   quadratic B-spline     src/Basis/bspline.jl:28-184 (fast full-support path and
//                          the nodewise path for truncated windows)
//   uGIMP                  src/Basis/gimp.jl:16-40
//   WLS (MLS-MPM)          src/Basis/wls.jl:22-84
// The basis values are evaluated inside the transfers ("deferred" weights,
// src/Transfer/runtime.jl:55-130), so no weight array crosses HBM.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/tesserae_b200.h"

namespace tb {

// Error bits a kernel raises in the context's device status word.
enum : int {
    ERR_TILE_RANGE = 1,   // a support window left its block tile
    ERR_GIMP_LENGTH = 2,  // uGIMP requires 0 <= l <= h (gimp.jl:22)
    ERR_WLS_SINGULAR = 4,  // WLS moment matrix not invertible
    ERR_REORDER_OUTSIDE = 8,  // a reorder was due but particles lie outside the mesh
    ERR_INACTIVE_NODE = 16,   // a scatter reached a node of an inactive block of a sparse grid
    ERR_SPGRID_CAPACITY = 32  // a sparse grid's active blocks exceed its field arrays
};

// CTAs that share one block of the block list: the average particle count of
// the non-empty blocks (totals = {nactive, nassigned}) over `per_cta`, the
// particles one CTA takes per pass, between 1 and 8. A crowded scene (4^3
// particles per cell: 4096 per 4^3-cell block) has fewer blocks than the GPU
// has CTA slots; splitting each block's passes over several CTAs (CTA `sub` of
// `split` takes passes sub, sub + split, ...) restores the parallelism. The
// transfers add each pass's tile to the grid with global atomics anyway, so
// the split costs no extra work.
__device__ __forceinline__ int block_split(const int* totals, int per_cta) {
    const long long nact = totals[0], nass = totals[1];
    if (nact <= 0) return 1;
    const long long s = (nass / nact + per_cta / 2) / per_cta;
    return int(s < 1 ? 1 : (s > 8 ? 8 : s));
}

// The passes of one block's particle range [s0, s1) for kernels that hold `per`
// particles (a multiple of 8) at a time: pass i of count() = ceil(n / per)
// takes the 8-particle chunks i, i + count(), i + 2 count(), ..., so every pass
// samples the whole block. A block denser than one pass whose particles lie in
// lattice order (4^3 per cell: 16 lattice rows of x per block row) would
// otherwise give each pass a few (y, z) rows of the block, all of its records
// to a few pencils, and a sweep as long as the longest of them. A 32-particle
// warp load touches 4 chunks of 8, the same sectors as a contiguous one for
// 4-byte fields. With one pass this is the range itself, in order.
struct BlockPasses {
    int s0, s1, npass;
    __device__ __forceinline__ BlockPasses(int a, int b, int per) : s0(a), s1(b), npass((b - a + per - 1) / per) {}
    __device__ __forceinline__ int count() const { return npass; }
    // position in the block list of item t (0 <= t < per) of pass i (>= s1: past the range)
    __device__ __forceinline__ int pos(int i, int t) const { return s0 + ((i + npass * (t >> 3)) << 3) + (t & 7); }
    // pos(i, t + nt) - pos(i, t) for nt a multiple of 8
    __device__ __forceinline__ int step(int nt) const { return npass * nt; }
};

// Forward-mode dual number with the three derivatives with respect to a
// particle's position: the weights evaluated in Dual3 give dN/dx_p and
// d(grad N)/dx_p for the reverse step of every basis (WLS, KernelCorrection,
// truncated windows) without hand-derived second derivatives. Floors and
// comparisons act on the value, |x| follows the value's sign. In a namespace of
// its own, so that floor, fabs and signbit of plain numbers inside tb still
// resolve to the CUDA functions (the Dual3 overloads are found by argument-
// dependent lookup).
namespace ad {
struct Dual3 {
    double v, d[3];
    __host__ __device__ Dual3() : v(0.0), d{0.0, 0.0, 0.0} {}
    __host__ __device__ Dual3(double a) : v(a), d{0.0, 0.0, 0.0} {}
    __host__ __device__ explicit operator double() const { return v; }
    __host__ __device__ explicit operator float() const { return float(v); }
    __host__ __device__ explicit operator int() const { return int(v); }
    __host__ __device__ Dual3 operator-() const {
        Dual3 r;
        r.v = -v;
        for (int k = 0; k < 3; ++k) r.d[k] = -d[k];
        return r;
    }
    __host__ __device__ Dual3& operator+=(const Dual3& o) {
        v += o.v;
        for (int k = 0; k < 3; ++k) d[k] += o.d[k];
        return *this;
    }
    __host__ __device__ Dual3& operator-=(const Dual3& o) {
        v -= o.v;
        for (int k = 0; k < 3; ++k) d[k] -= o.d[k];
        return *this;
    }
    __host__ __device__ Dual3& operator*=(const Dual3& o) {
        for (int k = 0; k < 3; ++k) d[k] = d[k] * o.v + v * o.d[k];
        v *= o.v;
        return *this;
    }
    __host__ __device__ Dual3& operator/=(const Dual3& o) {
        const double iv = 1.0 / o.v;
        for (int k = 0; k < 3; ++k) d[k] = (d[k] - v * iv * o.d[k]) * iv;
        v *= iv;
        return *this;
    }
};
__host__ __device__ inline Dual3 operator+(Dual3 a, const Dual3& b) { return a += b; }
__host__ __device__ inline Dual3 operator-(Dual3 a, const Dual3& b) { return a -= b; }
__host__ __device__ inline Dual3 operator*(Dual3 a, const Dual3& b) { return a *= b; }
__host__ __device__ inline Dual3 operator/(Dual3 a, const Dual3& b) { return a /= b; }
__host__ __device__ inline bool operator<(const Dual3& a, const Dual3& b) { return a.v < b.v; }
__host__ __device__ inline bool operator>(const Dual3& a, const Dual3& b) { return a.v > b.v; }
__host__ __device__ inline bool operator<=(const Dual3& a, const Dual3& b) { return a.v <= b.v; }
__host__ __device__ inline bool operator>=(const Dual3& a, const Dual3& b) { return a.v >= b.v; }
__host__ __device__ inline bool operator==(const Dual3& a, const Dual3& b) { return a.v == b.v; }
__host__ __device__ inline bool operator!=(const Dual3& a, const Dual3& b) { return a.v != b.v; }
__device__ inline Dual3 floor(const Dual3& a) { return Dual3(::floor(a.v)); }
__device__ inline Dual3 fabs(const Dual3& a) { return ::signbit(a.v) ? -a : a; }
__device__ inline bool signbit(const Dual3& a) { return ::signbit(a.v); }
}  // namespace ad
using ad::Dual3;

template <int D, class T>
struct DMesh {
    int n[3];      // nodes per axis
    int nb[3];     // blocks per axis
    int L;         // block_log2
    int nblocks;
    long long nnodes;
    T xmin[3];
    T h, h_inv;
    double xmin64[3], h64, h_inv64;
};

template <int D, class T>
inline DMesh<D, T> make_dmesh(const tb_mesh& m) {
    DMesh<D, T> M{};
    M.L = m.block_log2;
    M.nblocks = 1;
    M.nnodes = 1;
    for (int d = 0; d < 3; ++d) {
        M.n[d] = d < D ? int(m.n_nodes[d]) : 1;
        M.nb[d] = d < D ? ((M.n[d] - 1) >> M.L) + 1 : 1;
        M.xmin[d] = T(m.xmin[d]);
        M.xmin64[d] = m.xmin[d];
        M.nblocks *= M.nb[d];
        M.nnodes *= M.n[d];
    }
    M.h = T(m.h);          // the Float32 form casts h and h_inv separately (src/adapt.jl:53-57)
    M.h_inv = T(m.h_inv);
    M.h64 = m.h;
    M.h_inv64 = m.h_inv;
    return M;
}

// Particle SoA views. T is the state scalar; F is always double. In the
// FP64-position form (FP32 state with FP64 positions) x is NULL and x64 holds
// the positions; otherwise x64 is NULL.
template <class T>
struct PView {
    long long n;
    T* x[3];
    double* x64[3];
    T* v[3];
    T* V;
    const T* m;
    const T* l;
    T* gv[9];
    T* sig[6];
    double* F[9];
    T* B[9];
    const T* V0;
    const T* mu;
    const T* lam;
    T* eps_p;      // von Mises: equivalent plastic strain
    T* Cp_inv[6];  // von Mises: inverse plastic right Cauchy-Green tensor (symmetric)
    // Where G2P stores the new positions when they must not replace x yet
    // (G2P2G: its P2G half weighs at the old ones); NULL = in place.
    T* x_out[3];
    double* x64_out[3];
};

template <class T>
struct GView {
    T* m;
    T* mv[3];
    T* f[3];
    T* v[3];
    T* vn[3];
    // block-sparse grid (bnum set): node block numbering (0 inactive, k >= 1
    // storage block k), the node block of each storage block (1-based ids),
    // the active block count (device), the nodes the fields hold and log2 of
    // the block edge
    const int* bnum;
    const int* blist;
    const int* nact;
    long long cap;
    int L;
};

// Storage slot of node (x, y, z) (z = 0 in 2D): the column-major linear index
// on a dense grid; on a block-sparse grid (src/Grids/spindices.jl storageindex)
// (k - 1) blocklength + the node's column-major index inside its block, k the
// block's storage number. -1: the block is inactive; -2: past the fields'
// capacity.
template <int D, class T, class MT>
__device__ __forceinline__ long long grid_slot(const GView<T>& G, const MT& M, int x, int y, int z) {
    if (!G.bnum) return (long long)x + (long long)M.n[0] * ((long long)y + (D == 3 ? (long long)M.n[1] * z : 0ll));
    const int L = G.L, W = 1 << L, mk = W - 1;
    const int B = (x >> L) + M.nb[0] * ((y >> L) + (D == 3 ? M.nb[1] * (z >> L) : 0));
    const int k = G.bnum[B];
    if (k <= 0) return -1;
    const int q = (x & mk) + W * ((y & mk) + (D == 3 ? W * (z & mk) : 0));
    const long long sl = (long long)(k - 1) * (D == 3 ? W * W * W : W * W) + q;
    return sl < G.cap ? sl : -2;
}

// Adds one node's P2G sums (m, mv[D], f[D], gravity already in f) to the grid,
// one atomic per non-zero value. A non-zero sum for a node that a sparse grid
// does not store sets ERR_INACTIVE_NODE (update_sparsity! was not run for these
// positions: src/Transfer/runtime.jl:152-161) or ERR_SPGRID_CAPACITY.
template <int D, class T, class MT, class V>
__device__ __forceinline__ void grid_add(const GView<T>& G, const MT& M, int* err, int x, int y, int z,
                                         const V* val) {
    bool any = val[0] != V(0);
#pragma unroll
    for (int c = 1; c < 1 + 2 * D; ++c) any = any || val[c] != V(0);
    if (!any) return;
    const long long sl = grid_slot<D>(G, M, x, y, z);
    if (sl < 0) {
        atomicOr(err, sl == -1 ? ERR_INACTIVE_NODE : ERR_SPGRID_CAPACITY);
        return;
    }
    if (val[0] != V(0)) atomicAdd(G.m + sl, T(val[0]));
#pragma unroll
    for (int d = 0; d < D; ++d) {
        if (val[1 + d] != V(0)) atomicAdd(G.mv[d] + sl, T(val[1 + d]));
        if (val[1 + D + d] != V(0)) atomicAdd(G.f[d] + sl, T(val[1 + D + d]));
    }
}

// Step scalars, converted once to the state type.
template <class T>
struct Scalars {
    T dt, mass, V0, g[3], gimp_l, alpha;
    double dt64, V0_64, mu, lam, hardening, yield_stress;
    int basis, transfer, material, wall_mask, wall_layers;
};

template <class T>
inline Scalars<T> make_scalars(const tb_step_params& p) {
    Scalars<T> s{};
    s.dt = T(p.dt);
    s.mass = T(p.mass);
    s.V0 = T(p.V0);
    for (int d = 0; d < 3; ++d) s.g[d] = T(p.gravity[d]);
    s.gimp_l = T(p.gimp_l);
    s.alpha = T(p.flip_alpha);
    s.dt64 = p.dt;
    s.V0_64 = p.V0;
    s.mu = p.mu;
    s.lam = p.lambda;
    s.basis = p.basis;
    s.transfer = p.transfer;
    s.material = p.material;
    s.wall_mask = p.wall_mask;
    s.wall_layers = p.wall_layers;
    s.hardening = p.hardening;
    s.yield_stress = p.yield_stress;
    return s;
}

// Basis kinds whose support window is uGIMP's, and the KernelCorrection kinds.
__host__ __device__ inline bool basis_is_gimp(int basis) {
    return basis == TB_UGIMP || basis == TB_WLS_UGIMP || basis == TB_KC_UGIMP;
}
__host__ __device__ inline bool basis_is_kc(int basis) {
    return basis == TB_KC_BSPLINE_QUADRATIC || basis == TB_KC_UGIMP;
}

template <int D>
__host__ __device__ constexpr int nsym() { return D == 3 ? 6 : 3; }

// Index of (r, c) in Tensorial's symmetric independent-component order.
template <int D>
__host__ __device__ constexpr int symidx(int r, int c) {
    return (r >= c) ? (c * D - c * (c - 1) / 2 + (r - c)) : (r * D - r * (r - 1) / 2 + (c - r));
}

// Node coordinate X_d(i) = xmin + i h, rounded once in FP64 and cast to T
// (the reference stores the axes as Vector{T}(range(xmin; step=h, length=n))).
template <int D, class T>
__device__ __forceinline__ T node_coord(const DMesh<D, T>& M, int d, int i) {
    return T(__dadd_rn(M.xmin64[d], __dmul_rn(double(i), M.h64)));
}

// 1-based linear block id (0 = outside), cartesian.jl:271-285 + sub2ind.
template <int D, class T>
__device__ __forceinline__ int findblock(const DMesh<D, T>& M, const T* x) {
    int lin = 0;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
        T c = floor((x[d] - M.xmin[d]) * M.h_inv);
        if (!(c >= T(0) && c <= T(M.n[d] - 2))) return 0;
        lin = lin * M.nb[d] + (int(c) >> M.L);
    }
    return lin + 1;
}

// findblock of an FP64 position with the mesh's FP64 xmin and h_inv (the
// Float64 rule of cartesian.jl:271-285, as findblock<D, double>).
template <int D, class T>
__device__ __forceinline__ int findblock_x64(const DMesh<D, T>& M, const double* x) {
    int lin = 0;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
        const double c = floor((x[d] - M.xmin64[d]) * M.h_inv64);
        if (!(c >= 0.0 && c <= double(M.n[d] - 2))) return 0;
        lin = lin * M.nb[d] + (int(c) >> M.L);
    }
    return lin + 1;
}

// Per-axis basis data of one particle: window start/count and the 1-D jets.
template <class T>
struct Axis {
    int lo, cnt;
    T val[3], der[3];
};

// 1-D jets, forward-mode derivative through abs() as in the reference's AD.
template <class T>
__device__ __forceinline__ void jet_bspline_quadratic(T xi, T& val, T& der) {
    T s = signbit(xi) ? T(-1) : T(1);
    T a = fabs(xi);
    if (a < T(0.5)) {
        val = (T(3) - T(4) * (a * a)) / T(4);
        der = -(T(2) * a) * s;
    } else if (a < T(1.5)) {
        T t = T(3) - T(2) * a;
        val = (t * t) / T(8);
        der = -(t / T(2)) * s;
    } else {
        val = T(0);
        der = T(0);
    }
}

template <class T>
__device__ __forceinline__ void jet_ugimp(T xi, T l, T& val, T& der) {
    T s = signbit(xi) ? T(-1) : T(1);
    T a = fabs(xi);
    if (a < l / T(2)) {
        val = T(1) - (T(4) * (a * a) + l * l) / (T(4) * l);
        der = -(T(2) * a / l) * s;
    } else if (a < T(1) - l / T(2)) {
        val = T(1) - a;
        der = -s;
    } else if (a < T(1) + l / T(2)) {
        T t = T(1) + l / T(2) - a;
        val = (t * t) / (T(2) * l);
        der = -(t / l) * s;
    } else {
        val = T(0);
        der = T(0);
    }
}

// Fast full-support axis values (bspline.jl:90-100): t = fract(xi - 1/2),
// N = (1/2 - t + t^2/2, 1/2 + t - t^2, t^2/2), N' = (t - 1, 1 - 2t, t).
template <class T>
__device__ __forceinline__ void bspline_quadratic_poly(T t, T* v0, T* v1) {
    const T half = T(0.5);
    v0[0] = half + t * (T(-1) + t * half);
    v0[1] = half + t * (T(1) + t * T(-1));
    v0[2] = t * (t * half);
    v1[0] = T(-1) + t;
    v1[1] = T(1) + t * T(-2);
    v1[2] = t;
}

template <class T>
__device__ __forceinline__ void bspline_quadratic_axis(T xi, T* v0, T* v1) {
    T u = xi - T(0.5);
    T t = u - floor(u);
    bspline_quadratic_poly(t, v0, v1);
}

// Window and 1-D jets of one particle for B-spline / uGIMP kernels (the
// kernel part of WLS too). Returns false when the particle is outside the mesh
// (empty window, cartesian.jl:190-199). `full` reports a 3^D window.
// Support window of one particle: xi = (x - xmin) h_inv per axis, the clamped
// window start and node count per axis (supportnodes, bspline.jl:28-40 and
// cartesian.jl:190-199). Returns false when the particle is outside the mesh.
template <int D, class T>
__device__ __forceinline__ bool axis_window(const DMesh<D, T>& M, int basis, const T* x, T lnorm, T* xi, int* lo,
                                            int* cnt) {
    bool inside = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        xi[d] = (x[d] - M.xmin[d]) * M.h_inv;
        T c = floor(xi[d]);
        inside = inside && (c >= T(0) && c <= T(M.n[d] - 2));
    }
    if (!inside) return false;
    const bool gimp = basis_is_gimp(basis);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        int s, e;
        if (gimp) {
            T r = T(1) + lnorm / T(2);
            s = int(floor(xi[d] - r)) + 1;
            e = int(floor(xi[d] + r));
        } else {
            s = int(floor(xi[d] - T(0.5)));
            e = s + 2;
        }
        lo[d] = max(s, 0);
        cnt[d] = min(e, M.n[d] - 1) - lo[d] + 1;
    }
    return true;
}

template <int D, class T>
__device__ __forceinline__ bool axis_weights(const DMesh<D, T>& M, int basis, const T* x, T lnorm, Axis<T>* ax,
                                             bool& full) {
    T xi[3];
    int lo[3], cnt[3];
    if (!axis_window<D, T>(M, basis, x, lnorm, xi, lo, cnt)) return false;
    const bool gimp = basis_is_gimp(basis);
    full = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        ax[d].lo = lo[d];
        ax[d].cnt = cnt[d];
        full = full && (ax[d].cnt == 3);
    }
    if ((basis == TB_BSPLINE_QUADRATIC || basis == TB_KC_BSPLINE_QUADRATIC) && full) {
#pragma unroll
        for (int d = 0; d < D; ++d) bspline_quadratic_axis(xi[d], ax[d].val, ax[d].der);
        return true;
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            ax[d].val[k] = T(0);
            ax[d].der[k] = T(0);
            if (k < ax[d].cnt) {
                T xn = (x[d] - node_coord(M, d, ax[d].lo + k)) * M.h_inv;
                if (gimp) jet_ugimp(xn, lnorm, ax[d].val[k], ax[d].der[k]);
                else jet_bspline_quadratic(xn, ax[d].val[k], ax[d].der[k]);
            }
        }
    }
    return true;
}

// KernelCorrection(kernel) with its default MultiLinear polynomial on a
// support the mesh cuts (src/Basis/kernelcorrection.jl:13-64; a whole support
// keeps the plain kernel). Without a node filter the MultiLinear weighted
// least-squares fit of a separable kernel is one 1-D fit with P = (1, X_i - x_p)
// per axis (the moment matrix of the tensor-product polynomial under a product
// weight is the Kronecker product of the axis moment matrices), the
// decomposition the reference evaluates for B-splines (wls.jl:88-103, 177-192).
// Per axis the kernel values w_k become w_k (M^-1 P_k)[0] and their derivative
// w_k (M^-1 P_k)[1]; a whole B-spline axis takes the closed form
// M^-1 = diag(1, 4/h^2) (wls.jl:29-49). `r[d][k]` = X_k - x_p. The derivative is
// stored in units of xi (times h) like the plain jets. False for a singular fit.
template <int D, class T>
__device__ __forceinline__ bool kc_correct(const DMesh<D, T>& M, bool bspline, const T (&r)[3][3], Axis<T>* ax) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
        if (bspline && ax[d].cnt == 3) {
            const T c = T(4) / (M.h * M.h);
#pragma unroll
            for (int k = 0; k < 3; ++k) ax[d].der[k] = ax[d].val[k] * (c * r[d][k]) * M.h;
        } else {
            T S0 = T(0), S1 = T(0), S2 = T(0);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (k >= ax[d].cnt) continue;
                S0 += ax[d].val[k];
                S1 += ax[d].val[k] * r[d][k];
                S2 += ax[d].val[k] * r[d][k] * r[d][k];
            }
            const T det = S0 * S2 - S1 * S1;
            if (det == T(0)) return false;
            const T i00 = S2 / det, i01 = -S1 / det, i11 = S0 / det;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const T w = ax[d].val[k];
                ax[d].val[k] = k < ax[d].cnt ? w * (i00 + i01 * r[d][k]) : T(0);
                ax[d].der[k] = k < ax[d].cnt ? w * (i01 + i11 * r[d][k]) * M.h : T(0);
            }
        }
    }
    return true;
}

// Kernel value and gradient at window slot (i, j, k), product order of
// bspline.jl:133-142 / basis_weight.jl:49-60.
template <int D, class T>
__device__ __forceinline__ void node_weight(const DMesh<D, T>& M, const Axis<T>* ax, int i, int j, int k, T& w,
                                            T* dw) {
    if constexpr (D == 3) {
        T vx = ax[0].val[i], vy = ax[1].val[j], vz = ax[2].val[k];
        w = (vx * vy) * vz;
        dw[0] = ((ax[0].der[i] * vy) * vz) * M.h_inv;
        dw[1] = ((vx * ax[1].der[j]) * vz) * M.h_inv;
        dw[2] = ((vx * vy) * ax[2].der[k]) * M.h_inv;
    } else {
        T vx = ax[0].val[i], vy = ax[1].val[j];
        w = vx * vy;
        dw[0] = (ax[0].der[i] * vy) * M.h_inv;
        dw[1] = (vx * ax[1].der[j]) * M.h_inv;
    }
}

// WLS moment-matrix inverse (wls.jl:51-68); the closed form diag(1, 4/h^2) for a
// full quadratic B-spline support (wls.jl:29-49). Returns false if singular.
// `r[d][k]` = X_{lo+k} - x_p on axis d. The kernel weight is a product of axis
// factors and P = (1, X - x_p) has one axis per component, so
// M = sum_i w_i P_i P_i^T is built from the axis moments S0 = sum w, S1 = sum w r,
// S2 = sum w r^2: M00 = prod S0, M0a = S1_a prod_{d!=a} S0_d,
// Maa = S2_a prod_{d!=a} S0_d, Mab = S1_a S1_b prod_{d!=a,b} S0_d -- the
// reference's sum over the window's nodes, regrouped (equal to rounding).
// Slots beyond a truncated window have w = 0 and drop out.
template <int D, class T>
__device__ __forceinline__ bool wls_minv(const DMesh<D, T>& M, const Axis<T>* ax, const T (&r)[3][3], bool closed,
                                         T (&Mi)[D + 1][D + 1]) {
    constexpr int N = D + 1;
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
        for (int c = 0; c < N; ++c) Mi[a][c] = T(0);
    if (closed) {
        Mi[0][0] = T(1);
        T cval = T(4) / (M.h * M.h);
#pragma unroll
        for (int d = 1; d < N; ++d) Mi[d][d] = cval;
        return true;
    }
    T S0[3], S1[3], S2[3];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        S0[d] = S1[d] = S2[d] = T(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const T w = ax[d].val[k];
            S0[d] += w;
            S1[d] += w * r[d][k];
            S2[d] += (w * r[d][k]) * r[d][k];
        }
    }
    T A[N][2 * N];
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
        for (int c = 0; c < N; ++c) {
            // factor of axis d in entry (a, c): S2 if both index d, S1 if one does, else S0
            T v = T(1);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const int hits = (a == d + 1) + (c == d + 1);
                v *= hits == 2 ? S2[d] : (hits == 1 ? S1[d] : S0[d]);
            }
            A[a][c] = v;
            A[a][c + N] = (a == c) ? T(1) : T(0);
        }
    // Gauss-Jordan with partial pivoting on [M | I].
#pragma unroll
    for (int c = 0; c < N; ++c) {
        int p = c;
#pragma unroll
        for (int q = c + 1; q < N; ++q)
            if (fabs(A[q][c]) > fabs(A[p][c])) p = q;
        if (A[p][c] == T(0)) return false;
        if (p != c) {
#pragma unroll
            for (int k = 0; k < 2 * N; ++k) {
                T t = A[p][k];
                A[p][k] = A[c][k];
                A[c][k] = t;
            }
        }
        T inv = T(1) / A[c][c];
#pragma unroll
        for (int k = 0; k < 2 * N; ++k) A[c][k] *= inv;
#pragma unroll
        for (int q = 0; q < N; ++q)
            if (q != c) {
                T f = A[q][c];
#pragma unroll
                for (int k = 0; k < 2 * N; ++k) A[q][k] -= f * A[c][k];
            }
    }
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
        for (int c = 0; c < N; ++c) Mi[a][c] = A[a][c + N];
    return true;
}

// Basis state of one particle, ready for per-node evaluation in a transfer.
template <int D, class T>
struct Basis {
    Axis<T> ax[D];
    T Mi[D + 1][D + 1];
    bool wls;
};

// Prepare the basis of one particle. Returns false for an empty window.
template <int D, class T, bool ALLOW_WLS = true>
__device__ __forceinline__ bool prepare_basis(const DMesh<D, T>& M, int basis, const T* x, T l_abs,
                                              Basis<D, T>& B, int* err) {
    T lnorm = T(0);
    if (basis_is_gimp(basis)) {
        lnorm = l_abs / M.h;
        if (!(lnorm >= T(0) && lnorm <= T(1))) {
            atomicOr(err, ERR_GIMP_LENGTH);
            return false;
        }
    }
    bool full = false;
    if (!axis_weights<D, T>(M, basis, x, lnorm, B.ax, full)) return false;
    if (basis_is_kc(basis) && !full) {
        T r[3][3] = {};
#pragma unroll
        for (int d = 0; d < D; ++d)
#pragma unroll
            for (int k = 0; k < 3; ++k) r[d][k] = node_coord(M, d, B.ax[d].lo + k) - x[d];
        if (!kc_correct<D, T>(M, basis == TB_KC_BSPLINE_QUADRATIC, r, B.ax)) {
            atomicOr(err, ERR_WLS_SINGULAR);
            return false;
        }
    }
    B.wls = ALLOW_WLS && (basis == TB_WLS_BSPLINE_QUADRATIC || basis == TB_WLS_UGIMP);
    if constexpr (ALLOW_WLS) if (B.wls) {
        bool closed = (basis == TB_WLS_BSPLINE_QUADRATIC) && full;
        T r[3][3] = {};
        if (!closed) {
#pragma unroll
            for (int d = 0; d < D; ++d)
#pragma unroll
                for (int k = 0; k < 3; ++k) r[d][k] = node_coord(M, d, B.ax[d].lo + k) - x[d];
        }
        if (!wls_minv<D, T>(M, B.ax, r, closed, B.Mi)) {
            atomicOr(err, ERR_WLS_SINGULAR);
            return false;
        }
    }
    return true;
}

// FP64-position form: the window and the 1-D jets of a particle whose position
// is FP64. xi = (x - xmin) h_inv and the in-cell offsets are computed in FP64;
// only the offset from the window's first node, a number in [0, 3), is rounded
// to T before the jets are evaluated, so the weights carry T's relative
// precision of that offset rather than of the absolute coordinate. Window rules
// as axis_window (B-spline and uGIMP; WLS is not on this form).
template <int D, class T>
__device__ __forceinline__ bool axis_window_x64(const DMesh<D, T>& M, int basis, const double* x, double lnorm,
                                                double* xi, int* lo, int* cnt) {
    bool inside = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        xi[d] = (x[d] - M.xmin64[d]) * M.h_inv64;
        const double c = floor(xi[d]);
        inside = inside && (c >= 0.0 && c <= double(M.n[d] - 2));
    }
    if (!inside) return false;
    const bool gimp = basis_is_gimp(basis);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        int st, e;
        if (gimp) {
            const double r = 1.0 + lnorm / 2.0;
            st = int(floor(xi[d] - r)) + 1;
            e = int(floor(xi[d] + r));
        } else {
            st = int(floor(xi[d] - 0.5));
            e = st + 2;
        }
        lo[d] = max(st, 0);
        cnt[d] = min(e, M.n[d] - 1) - lo[d] + 1;
    }
    return true;
}

template <int D, class T, bool ALLOW_WLS = false>
__device__ __forceinline__ bool prepare_basis_x64(const DMesh<D, T>& M, int basis, const double* x, T l_abs,
                                                  Basis<D, T>& B, int* err) {
    double lnorm = 0.0;
    const bool gimp = basis_is_gimp(basis);
    if (gimp) {
        lnorm = double(l_abs) / M.h64;
        if (!(lnorm >= 0.0 && lnorm <= 1.0)) {
            atomicOr(err, ERR_GIMP_LENGTH);
            return false;
        }
    }
    double xi[3];
    int lo[3], cnt[3];
    if (!axis_window_x64<D, T>(M, basis, x, lnorm, xi, lo, cnt)) return false;
    B.wls = false;
    bool full = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        B.ax[d].lo = lo[d];
        B.ax[d].cnt = cnt[d];
        full = full && cnt[d] == 3;
    }
    // X_{lo+k} - x_p in FP64, rounded once to T (KernelCorrection and WLS)
    auto rel = [&](T (&r)[3][3]) {
#pragma unroll
        for (int d = 0; d < D; ++d)
#pragma unroll
            for (int k = 0; k < 3; ++k) r[d][k] = T(__dadd_rn(M.xmin64[d], __dmul_rn(double(lo[d] + k), M.h64)) - x[d]);
    };
    if (!gimp && full) {
        // the fast path's t = fract(xi - 1/2) is xi - 1/2 - lo, in [0, 1); kept
        // below 1 after rounding so that the jets stay on the FP64 window
#pragma unroll
        for (int d = 0; d < D; ++d) {
            T t = T(xi[d] - 0.5 - double(lo[d]));
            if (t >= T(1)) t = T(1) - T(1) / T(1 << 24);
            bspline_quadratic_poly(t, B.ax[d].val, B.ax[d].der);
        }
    } else {
        const T ln = T(lnorm);
#pragma unroll
        for (int d = 0; d < D; ++d) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                B.ax[d].val[k] = T(0);
                B.ax[d].der[k] = T(0);
                if (k < cnt[d]) {
                    const T xn = T(xi[d] - double(lo[d] + k));
                    if (gimp) jet_ugimp(xn, ln, B.ax[d].val[k], B.ax[d].der[k]);
                    else jet_bspline_quadratic(xn, B.ax[d].val[k], B.ax[d].der[k]);
                }
            }
        }
        if (basis_is_kc(basis) && !full) {
            T r[3][3] = {};
            rel(r);
            if (!kc_correct<D, T>(M, basis == TB_KC_BSPLINE_QUADRATIC, r, B.ax)) {
                atomicOr(err, ERR_WLS_SINGULAR);
                return false;
            }
        }
    }
    if constexpr (ALLOW_WLS) {
        B.wls = basis == TB_WLS_BSPLINE_QUADRATIC || basis == TB_WLS_UGIMP;
        if (B.wls) {
            const bool closed = basis == TB_WLS_BSPLINE_QUADRATIC && full;
            T r[3][3] = {};
            if (!closed) rel(r);
            if (!wls_minv<D, T>(M, B.ax, r, closed, B.Mi)) {
                atomicOr(err, ERR_WLS_SINGULAR);
                return false;
            }
        }
    }
    return true;
}

// w and grad w at window slot (i, j, k); `rel` = X_i - x_p per axis.
template <int D, class T>
__device__ __forceinline__ void eval_node(const DMesh<D, T>& M, const Basis<D, T>& B, int i, int j, int k,
                                          const T* rel, T& w, T* dw) {
    node_weight<D, T>(M, B.ax, i, j, k, w, dw);
    if (B.wls) {
        constexpr int N = D + 1;
        T P[N];
        P[0] = T(1);
#pragma unroll
        for (int d = 0; d < D; ++d) P[d + 1] = rel[d];
        T wq[N];
#pragma unroll
        for (int r = 0; r < N; ++r) {
            T acc = T(0);
#pragma unroll
            for (int c = 0; c < N; ++c) acc += B.Mi[r][c] * P[c];
            wq[r] = w * acc;
        }
        w = wq[0];
#pragma unroll
        for (int d = 0; d < D; ++d) dw[d] = wq[d + 1];
    }
}

// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations
// (Golub & Van Loan, Matrix Computations, 4th ed., Algorithms 8.5.1-8.5.3):
// A = V diag(e) V^T, eigenvectors in the columns of V; stops when the
// off-diagonal part falls below 1e-15 of the matrix norm (at most 20 sweeps).
__device__ __forceinline__ void sym_eigen3(double (&a)[3][3], double (&e)[3], double (&V)[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) V[r][c] = (r == c) ? 1.0 : 0.0;
    double fro = 0.0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) fro += a[r][c] * a[r][c];
    for (int sweep = 0; sweep < 20; ++sweep) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        if (off <= 1e-30 * fro) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            if (a[p][q] == 0.0) continue;
            const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double akp = a[k][p], akq = a[k][q];
                a[k][p] = c * akp - sn * akq;
                a[k][q] = sn * akp + c * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double apk = a[p][k], aqk = a[q][k];
                a[p][k] = c * apk - sn * aqk;
                a[q][k] = sn * apk + c * aqk;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - sn * vkq;
                V[k][q] = sn * vkp + c * vkq;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) e[k] = a[k][k];
}

// The von Mises update of the Taylor impact (docs/src/gpu.md:352-391), one
// particle, FP64 throughout: F = dF F is given. Hencky elasticity on the trial
// left Cauchy-Green tensor b = F Cp^-1 F^T; yield f = sqrt(3/2 tau'.tau') -
// (tau_y0 + H eps_p) on the principal Kirchhoff deviator; return map
// Delta gamma = f / (3 mu + H) along df/dtau in principal logarithmic
// stretches; pressure kappa log J / J with kappa = lambda + 2 mu / 3. Writes
// sigma, Cp^-1 = F^-1 b_e F^-T, eps_p and V = det(dF) V. The G2P kernels that
// call it are instantiated apart from the elastic ones.
template <class T>
__device__ __forceinline__ void vonmises_update(const PView<T>& P, const Scalars<T>& s, long long p,
                                             const double (&F)[3][3], double detdF, double lam, double mu,
                                             T* sig_out, T* V_out) {
    const double kappa = lam + 2.0 * mu / 3.0;
    const double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                     F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                     F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
    const double lJ = log(J);
    const double pr = kappa * lJ / J;
    double Cp[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) Cp[r][c] = double(P.Cp_inv[symidx<3>(r, c)][p]);
    double FC[3][3], b[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) acc += F[r][k] * Cp[k][c];
            FC[r][c] = acc;
        }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) acc += FC[r][k] * F[c][k];
            b[r][c] = acc;
        }
    double a[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) a[r][c] = 0.5 * (b[r][c] + b[c][r]);
    double ev[3], n[3][3];
    sym_eigen3(a, ev, n);
    double lst[3], tau_tr[3], tt = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        lst[q] = sqrt(ev[q]);
        tau_tr[q] = 2.0 * mu * log(lst[q]) - 2.0 * mu / 3.0 * lJ;
        tt += tau_tr[q] * tau_tr[q];
    }
    const double epn = double(P.eps_p[p]);
    const double nrm = sqrt(1.5 * tt);
    const double ftr = nrm - (s.yield_stress + s.hardening * epn);
    double dgam = 0.0, le[3], tau[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        le[q] = lst[q];
        tau[q] = tau_tr[q];
    }
    if (ftr > 0.0) {
        dgam = ftr / (3.0 * mu + s.hardening);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double deps = dgam * (1.5 * tau_tr[q] / nrm);
            le[q] = exp(log(lst[q]) - deps);
            tau[q] = tau_tr[q] - 2.0 * mu * deps;
        }
    }
    double Fi[3][3];
    Fi[0][0] = (F[1][1] * F[2][2] - F[1][2] * F[2][1]) / J;
    Fi[0][1] = (F[0][2] * F[2][1] - F[0][1] * F[2][2]) / J;
    Fi[0][2] = (F[0][1] * F[1][2] - F[0][2] * F[1][1]) / J;
    Fi[1][0] = (F[1][2] * F[2][0] - F[1][0] * F[2][2]) / J;
    Fi[1][1] = (F[0][0] * F[2][2] - F[0][2] * F[2][0]) / J;
    Fi[1][2] = (F[0][2] * F[1][0] - F[0][0] * F[1][2]) / J;
    Fi[2][0] = (F[1][0] * F[2][1] - F[1][1] * F[2][0]) / J;
    Fi[2][1] = (F[0][1] * F[2][0] - F[0][0] * F[2][1]) / J;
    Fi[2][2] = (F[0][0] * F[1][1] - F[0][1] * F[1][0]) / J;
    // Fi n_q: Cp^-1 = sum_q le_q^2 (Fi n_q) (x) (Fi n_q)
    double m[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) m[r][q] = Fi[r][0] * n[0][q] + Fi[r][1] * n[1][q] + Fi[r][2] * n[2][q];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c <= r; ++c) {
            double sg = 0.0, cp = 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                sg += (tau[q] / J + pr) * n[r][q] * n[c][q];
                cp += le[q] * le[q] * m[r][q] * m[c][q];
            }
            P.sig[symidx<3>(r, c)][p] = T(sg);
            if (sig_out) sig_out[symidx<3>(r, c)] = T(sg);
            P.Cp_inv[symidx<3>(r, c)][p] = T(cp);
        }
    P.eps_p[p] = T(epn + dgam);
    const T Vn = T(detdF * double(P.V[p]));
    P.V[p] = Vn;
    if (V_out) *V_out = Vn;
}

// FP64 particle kinematics and constitutive update (README.md:82-86):
// F = (I + dt grad_v) F, J = det F, sigma by Neo-Hookean or the weakly
// compressible fluid p = -K (J - 1), V = V0 J; or, in 3D, the von Mises model
// of the Taylor impact with V = det(I + dt grad_v) V (vonmises_update). F, J
// and log J stay in FP64.
template <int D, class T>
__device__ __forceinline__ void load_F(const PView<T>& P, long long p, double (&F)[3][3]) {
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
        for (int c = 0; c < D; ++c) F[r][c] = P.F[r + c * D][p];
}

// F is passed in (the caller chooses when to load it).
template <int D, class T, bool VM = false>
__device__ __forceinline__ void particle_update(const PView<T>& P, const Scalars<T>& s, long long p,
                                                const T (&gv)[3][3], const double (&F)[3][3]) {
    double Fn[3][3];
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
        for (int c = 0; c < D; ++c) {
            double a = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                double Ark = (r == k ? 1.0 : 0.0) + double(gv[r][k]) * s.dt64;
                a += Ark * F[k][c];
            }
            Fn[r][c] = a;
        }
    double J;
    if constexpr (D == 3)
        J = Fn[0][0] * (Fn[1][1] * Fn[2][2] - Fn[1][2] * Fn[2][1]) -
            Fn[0][1] * (Fn[1][0] * Fn[2][2] - Fn[1][2] * Fn[2][0]) +
            Fn[0][2] * (Fn[1][0] * Fn[2][1] - Fn[1][1] * Fn[2][0]);
    else
        J = Fn[0][0] * Fn[1][1] - Fn[0][1] * Fn[1][0];
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
        for (int c = 0; c < D; ++c) P.F[r + c * D][p] = Fn[r][c];
    const double mu = P.mu ? double(P.mu[p]) : s.mu;
    const double lam = P.lam ? double(P.lam[p]) : s.lam;
    if constexpr (D == 3 && VM) {
        {
            double dF[3][3];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) dF[r][c] = (r == c ? 1.0 : 0.0) + double(gv[r][c]) * s.dt64;
            const double detdF = dF[0][0] * (dF[1][1] * dF[2][2] - dF[1][2] * dF[2][1]) -
                                 dF[0][1] * (dF[1][0] * dF[2][2] - dF[1][2] * dF[2][0]) +
                                 dF[0][2] * (dF[1][0] * dF[2][1] - dF[1][1] * dF[2][0]);
            vonmises_update<T>(P, s, p, Fn, detdF, lam, mu, nullptr, nullptr);
            return;
        }
    }
    if (s.material == 1) {
        const double pr = lam * (J - 1.0);
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c <= r; ++c) P.sig[symidx<D>(r, c)][p] = T(r == c ? pr : 0.0);
    } else {
        // sigma = (mu (F F^T - I) + lambda log J I) / J, the division by J taken
        // once as a reciprocal (one rounding more than six divisions)
        const double lj = log(J);
        const double iJ = 1.0 / J;
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c <= r; ++c) {
                double b = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) b += Fn[r][k] * Fn[c][k];
                double sg = (mu * (b - (r == c ? 1.0 : 0.0)) + (r == c ? lam * lj : 0.0)) * iJ;
                P.sig[symidx<D>(r, c)][p] = T(sg);
            }
    }
    const double V0 = P.V0 ? double(P.V0[p]) : s.V0_64;
    P.V[p] = T(V0 * J);
}

}  // namespace tb
