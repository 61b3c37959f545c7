// tb_oracle.hpp -- CPU restatement of Tesserae.jl's explicit MPM step.
//
// TEST INFRASTRUCTURE ONLY. This header is the parity oracle for the CUDA
// kernels of libtesserae_b200.so and the timed CPU baseline of bench.py. Only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs
// load it. The product library never links it.
//
// It restates, templated on the dimension D and the state scalar T (F is
// always double, as in the mixed FP32 form), the reference's algorithm:
//   mesh / findblock / support windows   src/Mesh/cartesian.jl:146-285
//   quadratic B-spline, fast and nodewise src/Basis/bspline.jl:28-184
//   uGIMP                                 src/Basis/gimp.jl:16-40
//   WLS (MLS-MPM)                         src/Basis/wls.jl:22-84, polynomials.jl:28-29
//   KernelCorrection                      src/Basis/kernelcorrection.jl:13-64, wls.jl:86-117
//   von Mises plasticity (Taylor impact)  docs/src/gpu.md:202-392
//   stable block partition                src/Parallel/cpu_block_strategy.jl:62-190
//   P2G / grid update / G2P               README.md:71-87, docs/src/gpu.md:296-331,
//                                         test/transfer.jl:85-136
//   APIC                                  docs/src/transfer.md:166-186
//   colour-phased parallel scatter        src/Parallel/region.jl:212-256
//
// Parity of this restatement against the reference itself is pinned only by the
// reference's known-answer tests and doctests (Julia is not available to run the
// reference); see tests/golden/.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <type_traits>

#include "../include/tesserae_b200.h"

namespace tbo {

// ---------------------------------------------------------------------------
// forward-mode dual numbers: a value and one directional derivative, carried
// through the same templated step (T = Dual, with the FP64 kinematics in Dual
// too) to give directional derivatives of a rollout: the gradient check of the
// hand-written reverse step that stands in for differentiating the reference
// with ForwardDiff (which cannot run here). Floors and comparisons act on the
// value (piecewise constant), |x| and the kernels' branches follow the value,
// as ForwardDiff's Dual numbers do.
// ---------------------------------------------------------------------------

struct Dual {
    double v = 0.0, d = 0.0;
    Dual() = default;
    Dual(double a) : v(a), d(0.0) {}  // constants carry no derivative
    Dual(double a, double b) : v(a), d(b) {}
    explicit operator double() const { return v; }
    explicit operator float() const { return float(v); }
    explicit operator int64_t() const { return int64_t(v); }
    Dual operator-() const { return Dual(-v, -d); }
    Dual& operator+=(const Dual& o) { v += o.v; d += o.d; return *this; }
    Dual& operator-=(const Dual& o) { v -= o.v; d -= o.d; return *this; }
    Dual& operator*=(const Dual& o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
    Dual& operator/=(const Dual& o) { d = (d * o.v - v * o.d) / (o.v * o.v); v /= o.v; return *this; }
};
inline Dual operator+(Dual a, const Dual& b) { return a += b; }
inline Dual operator-(Dual a, const Dual& b) { return a -= b; }
inline Dual operator*(Dual a, const Dual& b) { return a *= b; }
inline Dual operator/(Dual a, const Dual& b) { return a /= b; }
inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
inline bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
inline bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }

template <class T> inline T floor_(T x) { return std::floor(x); }
template <class T> inline T fabs_(T x) { return std::fabs(x); }
template <class T> inline bool signbit_(T x) { return std::signbit(x); }
template <class T> inline T log_(T x) { return std::log(x); }
inline Dual floor_(Dual x) { return Dual(std::floor(x.v), 0.0); }
inline Dual fabs_(Dual x) { return std::signbit(x.v) ? -x : x; }
inline bool signbit_(Dual x) { return std::signbit(x.v); }
inline Dual log_(Dual x) { return Dual(std::log(x.v), x.d / x.v); }

// The type of the FP64 kinematics (F, det F, log J, the stress): double for the
// float and double forms, Dual for the dual form.
template <class T> struct Wide { using type = double; };
template <> struct Wide<Dual> { using type = Dual; };

// ---------------------------------------------------------------------------
// mesh
// ---------------------------------------------------------------------------

template <int D, class T>
struct Mesh {
    int64_t n[3];
    int64_t nb[3];
    T xmin[3];
    T h, h_inv;
    double xmin64[3], h64;  // FP64 originals for node coordinates
    int L;
    int64_t nnodes, nblocks;
};

template <int D, class T>
inline Mesh<D, T> make_mesh(const tb_mesh& m) {
    Mesh<D, T> M{};
    M.L = m.block_log2;
    M.nnodes = 1;
    M.nblocks = 1;
    for (int d = 0; d < 3; ++d) {
        M.n[d] = d < D ? m.n_nodes[d] : 1;
        // nblocks: ((n - 1) >> L) + 1 (src/Mesh/cartesian.jl:241-242)
        M.nb[d] = d < D ? ((M.n[d] - 1) >> M.L) + 1 : 1;
        M.xmin[d] = T(m.xmin[d]);
        M.xmin64[d] = m.xmin[d];
        M.nnodes *= M.n[d];
        M.nblocks *= M.nb[d];
    }
    // The Float32 form casts h and h_inv separately (src/adapt.jl:53-57).
    M.h = T(m.h);
    M.h_inv = T(m.h_inv);
    M.h64 = m.h;
    return M;
}

// Node coordinate on axis d, as the scalar type of the mesh axes. The reference
// stores axes as Vector{T}(range(xmin; step=h, length=n)) (cartesian.jl:86-101),
// xmin + i*h evaluated in Julia's TwicePrecision and rounded once; here it is
// xmin + i*h in FP64 (unfused), which agrees exactly when h is a power of two and
// to one ulp otherwise. The CUDA kernels use the same FP64 expression.
template <int D, class T>
inline T node_coord(const Mesh<D, T>& M, int d, int64_t i) {
    double x = M.xmin64[d] + double(i) * M.h64;
    return T(x);
}

template <int D>
inline int64_t node_linear(const int64_t* n, const int64_t* idx) {
    int64_t lin = idx[D - 1];
    for (int d = D - 2; d >= 0; --d) lin = lin * n[d] + idx[d];
    return lin;
}

// findblock: 1-based linear block id, 0 when outside (src/Mesh/cartesian.jl:271-285,
// gpu_block_strategy.jl:46-53 sub2ind). cell0 = trunc(floor((x - xmin) * h_inv)),
// inside iff 0 <= cell0 <= n - 2 on every axis.
template <int D, class T>
inline int32_t findblock(const Mesh<D, T>& M, const T* x) {
    int64_t b[3] = {0, 0, 0};
    for (int d = 0; d < D; ++d) {
        T c = floor_((x[d] - M.xmin[d]) * M.h_inv);
        if (!(c >= T(0) && c <= T(M.n[d] - 2))) return 0;
        b[d] = int64_t(c) >> M.L;
    }
    int64_t lin = b[D - 1];
    for (int d = D - 2; d >= 0; --d) lin = lin * M.nb[d] + b[d];
    return int32_t(lin + 1);
}

// ---------------------------------------------------------------------------
// basis
// ---------------------------------------------------------------------------

constexpr int NW3 = 27;

template <int D>
constexpr int nwin() { return D == 3 ? 27 : 9; }

template <int D, class T>
struct Weights {
    int64_t lo[3];   // 0-based first node per axis
    int64_t cnt[3];  // nodes per axis (0 = empty window)
    bool empty;
    T w[27];         // local slot s = i + 3 j + 9 k (column-major 3^D storage)
    T dw[27][3];
};

// 1-D jet of BSpline(Quadratic()) (src/Basis/bspline.jl:180-184, derivative by
// forward-mode AD through abs()). Known answer: jet(0) = (0.75, 0.0) (test/basis.jl:311).
template <class T>
inline void jet_bspline_quadratic(T xi, T& val, T& der) {
    T s = signbit_(xi) ? T(-1) : T(1);
    T a = fabs_(xi);
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

// 1-D jet of uGIMP with l normalised by h (src/Basis/gimp.jl:28-33).
template <class T>
inline void jet_ugimp(T xi, T l, T& val, T& der) {
    T s = signbit_(xi) ? T(-1) : T(1);
    T a = fabs_(xi);
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

// Normalised coordinate and the inside test of supportnodes (cartesian.jl:157-163,
// 227-234: floor(xi) in [0, n-2] on every axis).
template <int D, class T>
inline bool normalize_inside(const Mesh<D, T>& M, const T* x, T* xi) {
    bool inside = true;
    for (int d = 0; d < D; ++d) {
        xi[d] = (x[d] - M.xmin[d]) * M.h_inv;
        T c = floor_(xi[d]);
        inside = inside && (c >= T(0) && c <= T(M.n[d] - 2));
    }
    return inside;
}

// Quadratic B-spline window: start = trunc(floor(xi - 1/2)) + 1 (1-based), width 3,
// clipped to the mesh (src/Basis/bspline.jl:28-40).
template <int D, class T>
inline void window_bspline_quadratic(const Mesh<D, T>& M, const T* xi, Weights<D, T>& W) {
    for (int d = 0; d < 3; ++d) { W.lo[d] = 0; W.cnt[d] = 1; }
    for (int d = 0; d < D; ++d) {
        int64_t s = int64_t(floor_(xi[d] - T(1) / T(2)));
        int64_t e = s + 2;
        int64_t lo = std::max<int64_t>(s, 0), hi = std::min<int64_t>(e, M.n[d] - 1);
        W.lo[d] = lo;
        W.cnt[d] = hi - lo + 1;
    }
}

// uGIMP window: supportnodes(x, 1 + l/2, mesh), start = trunc(floor(xi - r)) + 2,
// stop = trunc(floor(xi + r)) + 1 (1-based) (src/Mesh/cartesian.jl:190-199, gimp.jl:20-24).
template <int D, class T>
inline void window_ugimp(const Mesh<D, T>& M, const T* xi, T lnorm, Weights<D, T>& W) {
    T r = T(1) + lnorm / T(2);
    for (int d = 0; d < 3; ++d) { W.lo[d] = 0; W.cnt[d] = 1; }
    for (int d = 0; d < D; ++d) {
        int64_t s = int64_t(floor_(xi[d] - r)) + 1;
        int64_t e = int64_t(floor_(xi[d] + r));
        int64_t lo = std::max<int64_t>(s, 0), hi = std::min<int64_t>(e, M.n[d] - 1);
        W.lo[d] = lo;
        W.cnt[d] = hi - lo + 1;
    }
}

template <int D, class T>
inline void zero_weights(Weights<D, T>& W) {
    for (int s = 0; s < 27; ++s) {
        W.w[s] = T(0);
        W.dw[s][0] = W.dw[s][1] = W.dw[s][2] = T(0);
    }
}

// Separable nodewise jet at every window node (basis_weight.jl:49-60, 625-632):
// xi_d = (x_d - X_d(i)) h_inv, w = prod vals, grad_d = (prod with der on axis d) * h_inv.
template <int D, class T, class Jet>
inline void nodewise_values(const Mesh<D, T>& M, const T* x, Weights<D, T>& W, Jet jet) {
    for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
        for (int j = 0; j < W.cnt[1]; ++j)
            for (int i = 0; i < W.cnt[0]; ++i) {
                int64_t node[3] = {W.lo[0] + i, W.lo[1] + j, W.lo[2] + k};
                int loc[3] = {i, j, k};
                T val[3], der[3];
                for (int d = 0; d < D; ++d) {
                    T xid = (x[d] - node_coord(M, d, node[d])) * M.h_inv;
                    jet(xid, val[d], der[d]);
                }
                int s = loc[0] + 3 * loc[1] + (D == 3 ? 9 * loc[2] : 0);
                T w = val[0];
                for (int d = 1; d < D; ++d) w = w * val[d];
                W.w[s] = w;
                for (int g = 0; g < D; ++g) {
                    T p = (g == 0 ? der[0] : val[0]);
                    for (int d = 1; d < D; ++d) p = p * (g == d ? der[d] : val[d]);
                    W.dw[s][g] = p * M.h_inv;
                }
            }
}

// Full-support fast path (bspline.jl:90-100, 146-170): t = fract(xi - 1/2),
// node values by Horner on the generated coefficients
//   N0 = 1/2 - t + t^2/2, N1 = 1/2 + t - t^2, N2 = t^2/2, N' = (-1 + t, 1 - 2t, t).
template <class T>
inline void bspline_quadratic_axis(T xi, T* v0, T* v1) {
    T u = xi - T(0.5);
    T t = u - floor_(u);
    const T half = T(1) / T(2);
    v0[0] = half + t * (T(-1) + t * half);
    v0[1] = half + t * (T(1) + t * T(-1));
    v0[2] = T(0) + t * (T(0) + t * half);
    v1[0] = T(-1) + t * T(1);
    v1[1] = T(1) + t * T(-2);
    v1[2] = T(0) + t * T(1);
}

template <int D, class T>
inline void fast_values(const Mesh<D, T>& M, const T* xi, Weights<D, T>& W) {
    T v0[3][3], v1[3][3];
    for (int d = 0; d < D; ++d) bspline_quadratic_axis(xi[d], v0[d], v1[d]);
    for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                int loc[3] = {i, j, k};
                int s = i + 3 * j + (D == 3 ? 9 * k : 0);
                T w = v0[0][i];
                for (int d = 1; d < D; ++d) w = w * v0[d][loc[d]];
                W.w[s] = w;
                for (int g = 0; g < D; ++g) {
                    T p = (g == 0 ? v1[0][i] : v0[0][i]);
                    for (int d = 1; d < D; ++d) p = p * (g == d ? v1[d][loc[d]] : v0[d][loc[d]]);
                    W.dw[s][g] = p * M.h_inv;
                }
            }
}

// Inverse of a small symmetric matrix by Gauss-Jordan with partial pivoting.
template <class T, int N>
inline bool invert(const T (&A)[N][N], T (&Ainv)[N][N]) {
    T a[N][2 * N];
    for (int r = 0; r < N; ++r)
        for (int c = 0; c < 2 * N; ++c) a[r][c] = c < N ? A[r][c] : (c - N == r ? T(1) : T(0));
    for (int c = 0; c < N; ++c) {
        int p = c;
        for (int r = c + 1; r < N; ++r)
            if (fabs_(a[r][c]) > fabs_(a[p][c])) p = r;
        if (a[p][c] == T(0)) return false;
        if (p != c)
            for (int k = 0; k < 2 * N; ++k) std::swap(a[p][k], a[c][k]);
        T inv = T(1) / a[c][c];
        for (int k = 0; k < 2 * N; ++k) a[c][k] *= inv;
        for (int r = 0; r < N; ++r)
            if (r != c) {
                T f = a[r][c];
                for (int k = 0; k < 2 * N; ++k) a[r][k] -= f * a[c][k];
            }
    }
    for (int r = 0; r < N; ++r)
        for (int c = 0; c < N; ++c) Ainv[r][c] = a[r][c + N];
    return true;
}

// WLS correction (wls.jl:51-84): P = [1; X_i - x_p], wq = w M^-1 P,
// w_wls = wq[0], grad w_wls = wq[1:D]. Full quadratic B-spline support uses the
// closed form M^-1 = diag(1, 4/h^2 I) (wls.jl:29-49).
template <int D, class T>
inline void wls_correct(const Mesh<D, T>& M, const T* x, Weights<D, T>& W, bool closed_form) {
    constexpr int N = D + 1;
    T Minv[N][N];
    for (int r = 0; r < N; ++r)
        for (int c = 0; c < N; ++c) Minv[r][c] = T(0);
    auto rel = [&](int s, int64_t* node, T* P) {
        P[0] = T(1);
        for (int d = 0; d < D; ++d) P[d + 1] = node_coord(M, d, node[d]) - x[d];
    };
    if (closed_form) {
        Minv[0][0] = T(1);
        T c = T(4) / (M.h * M.h);
        for (int d = 1; d < N; ++d) Minv[d][d] = c;
    } else {
        T Mm[N][N];
        for (int r = 0; r < N; ++r)
            for (int c = 0; c < N; ++c) Mm[r][c] = T(0);
        for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
            for (int j = 0; j < W.cnt[1]; ++j)
                for (int i = 0; i < W.cnt[0]; ++i) {
                    int s = i + 3 * j + (D == 3 ? 9 * k : 0);
                    int64_t node[3] = {W.lo[0] + i, W.lo[1] + j, W.lo[2] + k};
                    T P[N];
                    rel(s, node, P);
                    for (int r = 0; r < N; ++r)
                        for (int c = 0; c < N; ++c) Mm[r][c] += W.w[s] * P[r] * P[c];
                }
        if (!invert<T, N>(Mm, Minv)) {
            zero_weights(W);
            return;
        }
    }
    for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
        for (int j = 0; j < W.cnt[1]; ++j)
            for (int i = 0; i < W.cnt[0]; ++i) {
                int s = i + 3 * j + (D == 3 ? 9 * k : 0);
                int64_t node[3] = {W.lo[0] + i, W.lo[1] + j, W.lo[2] + k};
                T P[N];
                rel(s, node, P);
                T wq[N];
                for (int r = 0; r < N; ++r) {
                    T acc = T(0);
                    for (int c = 0; c < N; ++c) acc += Minv[r][c] * P[c];
                    wq[r] = W.w[s] * acc;
                }
                W.w[s] = wq[0];
                for (int d = 0; d < D; ++d) W.dw[s][d] = wq[d + 1];
            }
}

// KernelCorrection(kernel) with its default MultiLinear polynomial
// (src/Basis/kernelcorrection.jl:13-64): the plain kernel on a whole support
// (3 nodes on every axis), else the weighted least-squares fit with the
// MultiLinear polynomial (wls.jl:86-117). Without a node filter that fit of a
// separable kernel is exactly one 1-D fit with P = (1, X_i - x_p) per axis, the
// moment matrix of a tensor-product polynomial under a product weight being the
// Kronecker product of the axis moment matrices; the reference evaluates the
// B-spline case that way (wls.jl:88-103, 177-192). Per axis: a whole B-spline
// axis takes the closed form M^-1 = diag(1, 4/h^2) (wls.jl:29-49), otherwise
// M = sum w P P^T is inverted; the corrected value is w (M^-1 P)[0] and its
// derivative w (M^-1 P)[1] (the jet of P at 0, wls.jl:70-84). The node weight is
// the product of the axis values, its gradient the product with the derivative
// on one axis.
template <int D, class T>
inline bool kc_values(const Mesh<D, T>& M, const T* x, bool bspline, T lnorm, Weights<D, T>& W) {
    T val[3][3] = {}, der[3][3] = {};
    for (int d = 0; d < D; ++d) {
        T w[3] = {T(0), T(0), T(0)}, r[3] = {T(0), T(0), T(0)};
        for (int k = 0; k < W.cnt[d]; ++k) {
            const T X = node_coord(M, d, W.lo[d] + k);
            const T xn = (x[d] - X) * M.h_inv;
            T v, g;
            if (bspline) jet_bspline_quadratic(xn, v, g);
            else jet_ugimp(xn, lnorm, v, g);
            w[k] = v;
            r[k] = X - x[d];
        }
        if (bspline && W.cnt[d] == 3) {
            const T c = T(4) / (M.h * M.h);
            for (int k = 0; k < 3; ++k) {
                val[d][k] = w[k];
                der[d][k] = w[k] * (c * r[k]);
            }
        } else {
            T S0 = T(0), S1 = T(0), S2 = T(0);
            for (int k = 0; k < W.cnt[d]; ++k) {
                S0 += w[k];
                S1 += w[k] * r[k];
                S2 += w[k] * r[k] * r[k];
            }
            const T det = S0 * S2 - S1 * S1;
            if (det == T(0)) return false;
            const T i00 = S2 / det, i01 = -S1 / det, i11 = S0 / det;
            for (int k = 0; k < W.cnt[d]; ++k) {
                val[d][k] = w[k] * (i00 + i01 * r[k]);
                der[d][k] = w[k] * (i01 + i11 * r[k]);
            }
        }
    }
    for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
        for (int j = 0; j < W.cnt[1]; ++j)
            for (int i = 0; i < W.cnt[0]; ++i) {
                const int loc[3] = {i, j, k};
                const int s = i + 3 * j + (D == 3 ? 9 * k : 0);
                T w = val[0][i];
                for (int d = 1; d < D; ++d) w = w * val[d][loc[d]];
                W.w[s] = w;
                for (int g = 0; g < D; ++g) {
                    T q = (g == 0 ? der[0][i] : val[0][i]);
                    for (int d = 1; d < D; ++d) q = q * (g == d ? der[d][loc[d]] : val[d][loc[d]]);
                    W.dw[s][g] = q;
                }
            }
    return true;
}

// update_basis_weight! for one particle (basis_weight.jl:638-642).
template <int D, class T>
inline void compute_weights(const Mesh<D, T>& M, int basis, const T* x, T l_abs, Weights<D, T>& W) {
    zero_weights(W);
    T xi[3] = {0, 0, 0};
    bool inside = normalize_inside(M, x, xi);
    if (!inside) {
        W.empty = true;
        for (int d = 0; d < 3; ++d) { W.lo[d] = 0; W.cnt[d] = 0; }
        return;
    }
    W.empty = false;
    bool gimp = (basis == TB_UGIMP || basis == TB_WLS_UGIMP || basis == TB_KC_UGIMP);
    T lnorm = gimp ? l_abs / M.h : T(0);
    if (gimp) window_ugimp(M, xi, lnorm, W);
    else window_bspline_quadratic(M, xi, W);
    bool full = true;
    for (int d = 0; d < D; ++d) full = full && (W.cnt[d] == 3);
    if (basis == TB_KC_BSPLINE_QUADRATIC || basis == TB_KC_UGIMP) {
        if (full && basis == TB_KC_BSPLINE_QUADRATIC) fast_values(M, xi, W);
        else if (full) nodewise_values(M, x, W, [lnorm](T a, T& v, T& g) { jet_ugimp(a, lnorm, v, g); });
        else if (!kc_values(M, x, basis == TB_KC_BSPLINE_QUADRATIC, lnorm, W)) zero_weights(W);
    } else if (basis == TB_BSPLINE_QUADRATIC) {
        if (full) fast_values(M, xi, W);
        else nodewise_values(M, x, W, [](T a, T& v, T& g) { jet_bspline_quadratic(a, v, g); });
    } else if (basis == TB_WLS_BSPLINE_QUADRATIC) {
        nodewise_values(M, x, W, [](T a, T& v, T& g) { jet_bspline_quadratic(a, v, g); });
        wls_correct(M, x, W, full);
    } else {
        nodewise_values(M, x, W, [lnorm](T a, T& v, T& g) { jet_ugimp(a, lnorm, v, g); });
        if (basis == TB_WLS_UGIMP) wls_correct(M, x, W, false);
    }
}

// ---------------------------------------------------------------------------
// particle / grid views
// ---------------------------------------------------------------------------

template <class T>
inline T* P(void* p) { return static_cast<T*>(p); }
template <class T>
inline const T* CP(const void* p) { return static_cast<const T*>(p); }

template <int D>
constexpr int nsym() { return D == 3 ? 6 : 3; }
template <int D>
inline int symidx(int r, int c) {
    if (r < c) std::swap(r, c);
    return c * D - c * (c - 1) / 2 + (r - c);
}

// ---------------------------------------------------------------------------
// partition (stable counting sort)
// ---------------------------------------------------------------------------

template <int D, class T>
inline void bin(const Mesh<D, T>& M, const tb_particles& p, tb_partition& part, int64_t* nactive,
                int64_t* nassigned) {
    const int64_t n = p.n;
    std::vector<int32_t> cursor(M.nblocks, 0);
    std::fill(part.counts, part.counts + M.nblocks, 0);
    for (int64_t i = 0; i < n; ++i) {
        T x[3] = {0, 0, 0};
        for (int d = 0; d < D; ++d) x[d] = CP<T>(p.x[d])[i];
        int32_t b = findblock(M, x);
        part.blockids[i] = b;
        if (b) part.counts[b - 1] += 1;
    }
    int64_t acc = 0, na = 0;
    for (int64_t b = 0; b < M.nblocks; ++b) {
        part.offsets[b] = int32_t(acc);
        cursor[b] = int32_t(acc);
        if (part.counts[b]) part.blocklist[na++] = int32_t(b + 1);
        acc += part.counts[b];
    }
    part.offsets[M.nblocks] = int32_t(acc);
    for (int64_t i = 0; i < n; ++i) {
        int32_t b = part.blockids[i];
        if (b) part.particleindices[cursor[b - 1]++] = int32_t(i + 1);
    }
    *nactive = na;
    *nassigned = acc;
}

// ---------------------------------------------------------------------------
// P2G / grid update / G2P
// ---------------------------------------------------------------------------

template <class T>
inline T opt(const void* arr, int64_t i, double dflt) {
    return arr ? CP<T>(arr)[i] : T(dflt);
}

template <int D, class T>
struct ParticleIn {
    T x[3], v[3], V, m, l;
    T sig[3][3];
    T B[3][3];
};

template <int D, class T>
inline void load_particle(const tb_particles& p, const tb_step_params& prm, int64_t i, ParticleIn<D, T>& q) {
    for (int d = 0; d < 3; ++d) { q.x[d] = T(0); q.v[d] = T(0); }
    for (int d = 0; d < D; ++d) {
        q.x[d] = CP<T>(p.x[d])[i];
        q.v[d] = CP<T>(p.v[d])[i];
    }
    q.V = CP<T>(p.V)[i];
    q.m = opt<T>(p.m, i, prm.mass);
    q.l = opt<T>(p.l, i, prm.gimp_l);
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) {
            q.sig[r][c] = CP<T>(p.sigma[symidx<D>(r, c)])[i];
            q.B[r][c] = (prm.transfer == TB_TRANSFER_APIC) ? CP<T>(p.B[r + c * D])[i] : T(0);
        }
}

// Scatter of one particle into the grid fields (README.md:72-74, test/transfer.jl:96-97,
// docs/src/transfer.md:176-178).
template <int D, class T, class Acc>
inline void p2g_particle(const Mesh<D, T>& M, const tb_step_params& prm, const ParticleIn<D, T>& q,
                         T* gm, T* const* gmv, T* const* gf) {
    Weights<D, T> W;
    compute_weights(M, prm.basis, q.x, q.l, W);
    if (W.empty) return;
    const T dinv = T(4) / (M.h * M.h);  // D_p^-1 = inv(h^2/4 I) for the quadratic B-spline
    for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
        for (int j = 0; j < W.cnt[1]; ++j)
            for (int i = 0; i < W.cnt[0]; ++i) {
                int s = i + 3 * j + (D == 3 ? 9 * k : 0);
                int64_t node[3] = {W.lo[0] + i, W.lo[1] + j, W.lo[2] + k};
                int64_t I = node_linear<D>(M.n, node);
                T w = W.w[s];
                T wm = w * q.m;
                gm[I] += wm;
                T vv[3];
                for (int d = 0; d < D; ++d) vv[d] = q.v[d];
                if (prm.transfer == TB_TRANSFER_APIC) {
                    T dx[3];
                    for (int d = 0; d < D; ++d) dx[d] = node_coord(M, d, node[d]) - q.x[d];
                    for (int r = 0; r < D; ++r) {
                        T a = T(0);
                        for (int c = 0; c < D; ++c) a += q.B[r][c] * dinv * dx[c];
                        vv[r] += a;
                    }
                }
                for (int d = 0; d < D; ++d) gmv[d][I] += wm * vv[d];
                for (int r = 0; r < D; ++r) {
                    T a = T(0);
                    for (int c = 0; c < D; ++c) a += (-q.V * q.sig[r][c]) * W.dw[s][c];
                    gf[r][I] += a + wm * T(prm.gravity[r]);
                }
            }
}

template <int D, class T>
inline void zero_p2g_targets(const Mesh<D, T>& M, tb_grid& g) {
    std::fill(P<T>(g.m), P<T>(g.m) + M.nnodes, T(0));
    for (int d = 0; d < D; ++d) {
        std::fill(P<T>(g.mv[d]), P<T>(g.mv[d]) + M.nnodes, T(0));
        std::fill(P<T>(g.f[d]), P<T>(g.f[d]) + M.nnodes, T(0));
    }
}

template <int D, class T>
inline void p2g(const Mesh<D, T>& M, const tb_particles& p, tb_grid& g, const tb_step_params& prm) {
    zero_p2g_targets(M, g);
    T* gmv[3] = {nullptr, nullptr, nullptr};
    T* gf[3] = {nullptr, nullptr, nullptr};
    for (int d = 0; d < D; ++d) { gmv[d] = P<T>(g.mv[d]); gf[d] = P<T>(g.f[d]); }
    for (int64_t i = 0; i < p.n; ++i) {
        ParticleIn<D, T> q;
        load_particle<D, T>(p, prm, i, q);
        p2g_particle<D, T, void>(M, prm, q, P<T>(g.m), gmv, gf);
    }
}

// Grid half of @P2G (docs/src/gpu.md:309-310, guarded by !iszero(m)) and the
// slip-wall slices (gpu.md:313-316).
template <int D, class T>
inline void grid_update_node(const Mesh<D, T>& M, tb_grid& g, const tb_step_params& prm, int64_t I) {
    T m = P<T>(g.m)[I];
    T dt = T(prm.dt);
    for (int d = 0; d < D; ++d) {
        T vn = T(0), v = T(0);
        if (m != T(0)) {
            vn = P<T>(g.mv[d])[I] / m;
            v = vn + (dt * P<T>(g.f[d])[I]) / m;
        }
        P<T>(g.vn[d])[I] = vn;
        P<T>(g.v[d])[I] = v;
    }
    if (prm.wall_mask) {
        int64_t idx[3], r = I;
        for (int d = 0; d < D; ++d) { idx[d] = r % M.n[d]; r /= M.n[d]; }
        for (int d = 0; d < D; ++d) {
            bool lo = (prm.wall_mask >> (2 * d)) & 1, hi = (prm.wall_mask >> (2 * d + 1)) & 1;
            if ((lo && idx[d] < prm.wall_layers) || (hi && idx[d] >= M.n[d] - prm.wall_layers)) {
                P<T>(g.vn[d])[I] = T(0);
                P<T>(g.v[d])[I] = T(0);
            }
        }
    }
}

template <int D, class T>
inline void grid_update(const Mesh<D, T>& M, tb_grid& g, const tb_step_params& prm) {
    for (int64_t I = 0; I < M.nnodes; ++I) grid_update_node(M, g, prm, I);
}

// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations
// (Golub & Van Loan, Matrix Computations, 4th ed., Algorithms 8.5.1-8.5.3):
// A = V diag(e) V^T, the columns of V the eigenvectors. Sweeps stop when the
// off-diagonal part is below 1e-15 of the matrix norm, or after 20 sweeps.
inline void sym_eigen3(const double (&A)[3][3], double (&e)[3], double (&V)[3][3]) {
    double a[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            a[r][c] = A[r][c];
            V[r][c] = (r == c) ? 1.0 : 0.0;
        }
    double fro = 0.0;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) fro += a[r][c] * a[r][c];
    for (int sweep = 0; sweep < 20; ++sweep) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        if (off <= 1e-30 * fro) break;
        const int pq[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        for (const auto& ij : pq) {
            const int p = ij[0], q = ij[1];
            if (a[p][q] == 0.0) continue;
            // the rotation (c, s) that zeroes a[p][q] (sym.schur2)
            const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs_(theta) + std::sqrt(theta * theta + 1.0));
            const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
            // a <- J^T a J, V <- V J with J = rotation in the (p, q) plane
            for (int k = 0; k < 3; ++k) {
                const double akp = a[k][p], akq = a[k][q];
                a[k][p] = c * akp - sn * akq;
                a[k][q] = sn * akp + c * akq;
            }
            for (int k = 0; k < 3; ++k) {
                const double apk = a[p][k], aqk = a[q][k];
                a[p][k] = c * apk - sn * aqk;
                a[q][k] = sn * apk + c * aqk;
            }
            for (int k = 0; k < 3; ++k) {
                const double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - sn * vkq;
                V[k][q] = sn * vkp + c * vkq;
            }
        }
    }
    for (int k = 0; k < 3; ++k) e[k] = a[k][k];
}

// The von Mises model of the Taylor impact (docs/src/gpu.md:362-391):
// Hencky elasticity on the trial left Cauchy-Green tensor b = F Cp^-1 F^T,
// yield f = sqrt(3/2 tau'.tau') - (tau_y0 + H eps_p) on the principal Kirchhoff
// deviator, return map Delta gamma = f / (3 mu + H) along df/dtau in principal
// logarithmic stretches, pressure kappa log J / J with kappa = lambda + 2 mu / 3;
// returns the Cauchy stress and the updated Cp^-1 = F^-1 b_e F^-T and eps_p.
inline void vonmises_model(const double (&Cpinv)[3][3], double epn, const double (&F)[3][3], double lam,
                           double mu, double H, double ty0, double (&sig)[3][3], double (&Cpinv_new)[3][3],
                           double& ep_new) {
    const double kappa = lam + 2.0 * mu / 3.0;
    const double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                     F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                     F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
    const double lJ = std::log(J);
    const double pr = kappa * lJ / J;
    double FC[3][3] = {}, b[3][3] = {};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k) FC[r][c] += F[r][k] * Cpinv[k][c];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k) b[r][c] += FC[r][k] * F[c][k];
    double bs[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) bs[r][c] = 0.5 * (b[r][c] + b[c][r]);
    double ev[3], n[3][3];
    sym_eigen3(bs, ev, n);
    double lst[3], tau[3], tau_tr[3];
    double tt = 0.0;
    for (int a = 0; a < 3; ++a) {
        lst[a] = std::sqrt(ev[a]);
        tau_tr[a] = 2.0 * mu * std::log(lst[a]) - 2.0 * mu / 3.0 * lJ;
        tt += tau_tr[a] * tau_tr[a];
    }
    const double nrm = std::sqrt(1.5 * tt);
    const double ftr = nrm - (ty0 + H * epn);
    double dgam = 0.0, le[3];
    for (int a = 0; a < 3; ++a) {
        le[a] = lst[a];
        tau[a] = tau_tr[a];
    }
    if (ftr > 0.0) {
        dgam = ftr / (3.0 * mu + H);
        for (int a = 0; a < 3; ++a) {
            const double deps = dgam * (1.5 * tau_tr[a] / nrm);
            le[a] = std::exp(std::log(lst[a]) - deps);
            tau[a] = tau_tr[a] - 2.0 * mu * deps;
        }
    }
    double be[3][3] = {};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a) {
                be[r][c] += le[a] * le[a] * n[r][a] * n[c][a];
                sig[r][c] = 0.0;
            }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a) sig[r][c] += (tau[a] / J + pr) * n[r][a] * n[c][a];
    // F^-1 by cofactors
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
    double Fb[3][3] = {}, C[3][3] = {};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k) Fb[r][c] += Fi[r][k] * be[k][c];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k) C[r][c] += Fb[r][k] * Fi[c][k];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Cpinv_new[r][c] = 0.5 * (C[r][c] + C[c][r]);
    ep_new = epn + dgam;
}

// One particle of @G2P (README.md:79-86, test/transfer.jl:112-136, transfer.md:180-184):
// FLIP/PIC blend or APIC, then F = (I + dt grad v) F in FP64, J = det F,
// Neo-Hookean sigma = (mu (F F^T - I) + lambda log J I) / J, V = V0 J.
template <int D, class T>
inline void g2p_particle(const Mesh<D, T>& M, const tb_grid& g, tb_particles& p, const tb_step_params& prm,
                         int64_t i) {
    T x[3] = {0, 0, 0}, vp[3] = {0, 0, 0};
    for (int d = 0; d < D; ++d) { x[d] = P<T>(p.x[d])[i]; vp[d] = P<T>(p.v[d])[i]; }
    T l = opt<T>(p.l, i, prm.gimp_l);
    Weights<D, T> W;
    compute_weights(M, prm.basis, x, l, W);
    T vpic[3] = {0, 0, 0}, dvflip[3] = {0, 0, 0}, gv[3][3] = {}, dx[3] = {0, 0, 0}, Bn[3][3] = {};
    const T dt = T(prm.dt);
    if (!W.empty) {
        for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
            for (int j = 0; j < W.cnt[1]; ++j)
                for (int ii = 0; ii < W.cnt[0]; ++ii) {
                    int s = ii + 3 * j + (D == 3 ? 9 * k : 0);
                    int64_t node[3] = {W.lo[0] + ii, W.lo[1] + j, W.lo[2] + k};
                    int64_t I = node_linear<D>(M.n, node);
                    T w = W.w[s];
                    T vi[3], vni[3];
                    for (int d = 0; d < D; ++d) {
                        vi[d] = CP<T>(g.v[d])[I];
                        vni[d] = CP<T>(g.vn[d])[I];
                    }
                    for (int d = 0; d < D; ++d) {
                        vpic[d] += w * vi[d];
                        dvflip[d] += w * (vi[d] - vni[d]);
                        dx[d] += (w * vi[d]) * dt;
                    }
                    for (int r = 0; r < D; ++r)
                        for (int c = 0; c < D; ++c) gv[r][c] += vi[r] * W.dw[s][c];
                    if (prm.transfer == TB_TRANSFER_APIC) {
                        T rel[3];
                        for (int d = 0; d < D; ++d) rel[d] = node_coord(M, d, node[d]) - x[d];
                        for (int r = 0; r < D; ++r)
                            for (int c = 0; c < D; ++c) Bn[r][c] += (w * vi[r]) * rel[c];
                    }
                }
    }
    if (prm.transfer == TB_TRANSFER_APIC) {
        for (int d = 0; d < D; ++d) P<T>(p.v[d])[i] = vpic[d];
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) P<T>(p.B[r + c * D])[i] = Bn[r][c];
    } else {
        const T a = T(prm.flip_alpha);
        for (int d = 0; d < D; ++d) {
            T vflip = vp[d] + dvflip[d];
            P<T>(p.v[d])[i] = (a == T(1)) ? vflip : (T(1) - a) * vpic[d] + a * vflip;
        }
    }
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) P<T>(p.grad_v[r + c * D])[i] = gv[r][c];
    for (int d = 0; d < D; ++d) P<T>(p.x[d])[i] = x[d] + dx[d];

    // FP64 kinematics and constitutive update (TD = double; Dual in the dual form).
    using TD = typename Wide<T>::type;
    TD F[3][3], Fn[3][3];
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) F[r][c] = CP<TD>(p.F[r + c * D])[i];
    const double dtd = prm.dt;
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) {
            TD a = 0.0;
            for (int k = 0; k < D; ++k) {
                TD Ark = TD(r == k ? 1.0 : 0.0) + TD(gv[r][k]) * TD(dtd);
                a += Ark * F[k][c];
            }
            Fn[r][c] = a;
        }
    TD J;
    if (D == 3)
        J = Fn[0][0] * (Fn[1][1] * Fn[2][2] - Fn[1][2] * Fn[2][1]) -
            Fn[0][1] * (Fn[1][0] * Fn[2][2] - Fn[1][2] * Fn[2][0]) +
            Fn[0][2] * (Fn[1][0] * Fn[2][1] - Fn[1][1] * Fn[2][0]);
    else
        J = Fn[0][0] * Fn[1][1] - Fn[0][1] * Fn[1][0];
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) P<TD>(p.F[r + c * D])[i] = Fn[r][c];
    const TD mu = p.mu ? TD(CP<T>(p.mu)[i]) : TD(prm.mu);
    const TD lam = p.lambda ? TD(CP<T>(p.lambda)[i]) : TD(prm.lambda);
    TD sig[3][3] = {};
    if (prm.material == TB_MATERIAL_VONMISES) {
        // docs/src/gpu.md:352-358: F = dF F, von Mises state update, V = det(dF) V
        if constexpr (D == 3 && std::is_same_v<TD, double>) {
            double Cp[3][3], Cpn[3][3], epn = double(CP<T>(p.eps_p)[i]), epo;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) Cp[r][c] = double(CP<T>(p.Cp_inv[symidx<D>(r, c)])[i]);
            vonmises_model(Cp, epn, Fn, lam, mu, prm.hardening, prm.yield_stress, sig, Cpn, epo);
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c <= r; ++c) {
                    P<T>(p.sigma[symidx<D>(r, c)])[i] = T(sig[r][c]);
                    P<T>(p.Cp_inv[symidx<D>(r, c)])[i] = T(Cpn[r][c]);
                }
            P<T>(p.eps_p)[i] = T(epo);
            double dF[3][3];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) dF[r][c] = (r == c ? 1.0 : 0.0) + double(gv[r][c]) * dtd;
            const double jd = dF[0][0] * (dF[1][1] * dF[2][2] - dF[1][2] * dF[2][1]) -
                              dF[0][1] * (dF[1][0] * dF[2][2] - dF[1][2] * dF[2][0]) +
                              dF[0][2] * (dF[1][0] * dF[2][1] - dF[1][1] * dF[2][0]);
            P<T>(p.V)[i] = T(jd * double(CP<T>(p.V)[i]));
        }
        return;
    }
    if (prm.material == 1) {
        for (int d = 0; d < D; ++d) sig[d][d] = lam * (J - TD(1.0));
    } else {
        const TD lj = log_(J);
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                TD b = 0.0;
                for (int k = 0; k < D; ++k) b += Fn[r][k] * Fn[c][k];
                sig[r][c] = (mu * (b - TD(r == c ? 1.0 : 0.0)) + (r == c ? lam * lj : TD(0.0))) / J;
            }
    }
    for (int r = 0; r < D; ++r)
        for (int c = 0; c <= r; ++c) P<T>(p.sigma[symidx<D>(r, c)])[i] = T(sig[r][c]);
    const TD V0 = p.V0 ? TD(CP<T>(p.V0)[i]) : TD(prm.V0);
    P<T>(p.V)[i] = T(V0 * J);
}

template <int D, class T>
inline void g2p(const Mesh<D, T>& M, const tb_grid& g, tb_particles& p, const tb_step_params& prm) {
    for (int64_t i = 0; i < p.n; ++i) g2p_particle(M, g, p, prm, i);
}

// ---------------------------------------------------------------------------
// reverse mode of one step (the reference has no adjoint; this differentiates
// the forward step above by hand, all adjoint arithmetic in double)
// ---------------------------------------------------------------------------

// Second derivatives of the 1-D kernels with respect to xi (the jets above
// differentiated once more, piece by piece).
inline double d2_bspline_quadratic(double xi) {
    const double a = std::fabs(xi);
    if (a < 0.5) return -2.0;
    if (a < 1.5) return 1.0;
    return 0.0;
}
inline double d2_ugimp(double xi, double l) {
    const double a = std::fabs(xi);
    if (a < l / 2) return -2.0 / l;
    if (a < 1.0 - l / 2) return 0.0;
    if (a < 1.0 + l / 2) return 1.0 / l;
    return 0.0;
}

// Value, gradient and Hessian (with respect to x_p) of the kernel at every
// window slot, from per-axis nodewise jets in double.
template <int D>
struct AdjWeights {
    double w[27], g[27][3], H[27][3][3];
};

template <int D, class T>
inline void adjoint_weights(const Mesh<D, T>& M, int basis, const T* x, T l_abs, const Weights<D, T>& W,
                            AdjWeights<D>& A) {
    const bool gimp = basis == TB_UGIMP;
    const double lnorm = gimp ? double(T(l_abs / M.h)) : 0.0;
    const double hi = double(M.h_inv);
    double val[3][3] = {}, der[3][3] = {}, d2[3][3] = {};
    for (int d = 0; d < D; ++d)
        for (int k = 0; k < W.cnt[d]; ++k) {
            const double xi = (double(x[d]) - double(node_coord(M, d, W.lo[d] + k))) * hi;
            if (gimp) {
                jet_ugimp(xi, lnorm, val[d][k], der[d][k]);
                d2[d][k] = d2_ugimp(xi, lnorm);
            } else {
                jet_bspline_quadratic(xi, val[d][k], der[d][k]);
                d2[d][k] = d2_bspline_quadratic(xi);
            }
        }
    for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
        for (int j = 0; j < W.cnt[1]; ++j)
            for (int i = 0; i < W.cnt[0]; ++i) {
                const int s = i + 3 * j + (D == 3 ? 9 * k : 0);
                const int loc[3] = {i, j, k};
                double w = 1.0;
                for (int d = 0; d < D; ++d) w *= val[d][loc[d]];
                A.w[s] = w;
                for (int a = 0; a < D; ++a) {
                    double g = der[a][loc[a]];
                    for (int c = 0; c < D; ++c)
                        if (c != a) g *= val[c][loc[c]];
                    A.g[s][a] = g * hi;
                    for (int b = 0; b < D; ++b) {
                        double h = (a == b) ? d2[a][loc[a]] : der[a][loc[a]] * der[b][loc[b]];
                        for (int c = 0; c < D; ++c)
                            if (c != a && c != b) h *= val[c][loc[c]];
                        A.H[s][a][b] = h * hi * hi;
                    }
                }
            }
}

inline bool adjoint_supported(const tb_step_params& prm) {
    return (prm.basis == TB_BSPLINE_QUADRATIC || prm.basis == TB_UGIMP) && prm.transfer == TB_TRANSFER_FLIP &&
           prm.material != TB_MATERIAL_VONMISES;
}

template <int D>
inline double det_and_cof(const double (&F)[3][3], double (&C)[3][3]) {
    if (D == 3) {
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
    }
    C[0][0] = F[1][1];
    C[0][1] = -F[1][0];
    C[1][0] = -F[0][1];
    C[1][1] = F[0][0];
    return F[0][0] * F[1][1] - F[0][1] * F[1][0];
}

// Sensitivity of the loss to F, mu and lambda through sigma(F) and V = V0 det F
// (Neo-Hookean sigma = (mu (F F^T - I) + lambda log J I) / J, or the fluid
// sigma = lambda (J - 1) I), given sigma_bar (full D x D) and V_bar.
template <int D>
inline void constitutive_adjoint(const double (&F)[3][3], double mu, double lam, double V0, int material,
                                 const double (&sb)[3][3], double Vb, double (&Fb)[3][3], double& mub,
                                 double& lamb) {
    double C[3][3] = {};
    const double J = det_and_cof<D>(F, C);
    double Jb = V0 * Vb;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Fb[r][c] = 0.0;
    mub = 0.0;
    lamb = 0.0;
    if (material == 1) {
        double tr = 0.0;
        for (int d = 0; d < D; ++d) tr += sb[d][d];
        lamb += (J - 1.0) * tr;
        Jb += lam * tr;
    } else {
        const double lj = std::log(J);
        double Bm[3][3] = {}, tau[3][3] = {};
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                double b = 0.0;
                for (int k = 0; k < D; ++k) b += F[r][k] * F[c][k];
                Bm[r][c] = b - (r == c ? 1.0 : 0.0);
                tau[r][c] = mu * Bm[r][c] + (r == c ? lam * lj : 0.0);
            }
        double st = 0.0, trt = 0.0;
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                st += sb[r][c] * tau[r][c];
                mub += (sb[r][c] / J) * Bm[r][c];
            }
        for (int d = 0; d < D; ++d) trt += sb[d][d] / J;
        Jb += -st / (J * J) + lam * trt / J;
        lamb += lj * trt;
        // F_bar += (B_bar + B_bar^T) F with B_bar = mu sigma_bar / J
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                double a = 0.0;
                for (int k = 0; k < D; ++k) a += (mu / J) * (sb[r][k] + sb[k][r]) * F[k][c];
                Fb[r][c] += a;
            }
    }
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) Fb[r][c] += Jb * C[r][c];
}

// ---- reverse step for every basis and the APIC transfer ---------------------
// The weights' position derivatives come from the weights themselves evaluated
// in dual numbers (one pass per axis of x_p), so WLS, KernelCorrection and the
// truncated windows need no hand-derived derivative: dN[s][a] = dN_s/dx_p,a and
// dG[s][c][a] = d(grad N_s)_c / dx_p,a.
template <int D>
struct GenAdjWeights {
    double w[27], g[27][3], dN[27][3], dG[27][3][3];
};

template <int D, class T>
inline void general_adjoint_weights(const tb_mesh& m, int basis, const T* x, T l_abs, const Weights<D, T>& W,
                                    GenAdjWeights<D>& A) {
    const Mesh<D, Dual> MD = make_mesh<D, Dual>(m);
    for (int s = 0; s < 27; ++s) {
        A.w[s] = double(W.w[s]);
        for (int c = 0; c < 3; ++c) A.g[s][c] = double(W.dw[s][c]);
    }
    for (int a = 0; a < D; ++a) {
        Dual xd[3];
        for (int d = 0; d < 3; ++d) xd[d] = Dual(double(x[d]), d == a ? 1.0 : 0.0);
        Weights<D, Dual> WD;
        compute_weights(MD, basis, xd, Dual(double(l_abs)), WD);
        for (int s = 0; s < 27; ++s) {
            A.dN[s][a] = WD.w[s].d;
            for (int c = 0; c < 3; ++c) A.dG[s][c][a] = WD.dw[s][c].d;
        }
    }
}

inline bool general_adjoint_supported(const tb_step_params& prm) {
    return prm.basis >= TB_BSPLINE_QUADRATIC && prm.basis <= TB_KC_UGIMP &&
           (prm.transfer == TB_TRANSFER_FLIP || prm.transfer == TB_TRANSFER_APIC) &&
           prm.material != TB_MATERIAL_VONMISES;
}

// One step backwards for any supported basis with the FLIP/PIC or APIC transfer.
// Forward (README.md:71-87, docs/src/transfer.md:166-186):
//   m_i = sum N m_p,  mv_i = sum N m_p u_ip (u = v_p, APIC: v_p + B_p D^-1 r_ip, r = x_i - x_p),
//   f_i = sum (-V_p sigma_p grad N + N m_p g);  grid half;  then per particle
//   v_pic = sum N v_i, L = sum v_i (x) grad N, x' = x + dt v_pic, F' = (I + dt L) F,
//   FLIP: v' = (1 - a) v_pic + a (v_p + sum N (v_i - vn_i));  APIC: v' = v_pic,
//   B' = sum N v_i (x) r.   `a.B` (APIC) carries the sensitivity to B.
template <int D, class T>
inline int adjoint_step_general(const tb_mesh& mraw, const Mesh<D, T>& M, tb_particles& p, tb_grid& g,
                                const tb_step_params& prm, tb_adjoint& a) {
    if (!general_adjoint_supported(prm)) return TB_ERR_UNSUPPORTED;
    const bool apic = prm.transfer == TB_TRANSFER_APIC;
    if (apic)
        for (int k = 0; k < D * D; ++k)
            if (!a.B[k] || !p.B[k]) return TB_ERR_ARG;
    p2g<D, T>(M, p, g, prm);
    grid_update<D, T>(M, g, prm);
    const int64_t nn = M.nnodes;
    const size_t ndn = static_cast<size_t>(D) * static_cast<size_t>(nn);
    std::vector<double> vb(ndn, 0.0), vnb(ndn, 0.0), pb(ndn, 0.0), fb(ndn, 0.0);
    std::vector<double> mb(static_cast<size_t>(nn), 0.0);
    const double dt = prm.dt, alpha = prm.flip_alpha;
    const double dinv = 4.0 / (double(M.h) * double(M.h));
    auto for_nodes = [&](const Weights<D, T>& W, auto&& fn) {
        if (W.empty) return;
        for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
            for (int j = 0; j < W.cnt[1]; ++j)
                for (int ii = 0; ii < W.cnt[0]; ++ii) {
                    const int s = ii + 3 * j + (D == 3 ? 9 * k : 0);
                    int64_t node[3] = {W.lo[0] + ii, W.lo[1] + j, W.lo[2] + k};
                    fn(s, node_linear<D>(M.n, node), node);
                }
    };
    // ---- G2P backwards
    for (int64_t i = 0; i < p.n; ++i) {
        T x[3] = {0, 0, 0};
        for (int d = 0; d < D; ++d) x[d] = CP<T>(p.x[d])[i];
        const T l = opt<T>(p.l, i, prm.gimp_l);
        Weights<D, T> W;
        compute_weights(M, prm.basis, x, l, W);
        GenAdjWeights<D> A{};
        if (!W.empty) general_adjoint_weights(mraw, prm.basis, x, l, W, A);
        double L[3][3] = {};
        for_nodes(W, [&](int s, int64_t I, const int64_t*) {
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) L[r][c] += double(CP<T>(g.v[r])[I]) * A.g[s][c];
        });
        double F[3][3] = {}, Fb[3][3] = {};
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                F[r][c] = CP<double>(p.F[r + c * D])[i];
                Fb[r][c] = a.F[r + c * D][i];
            }
        double Lb[3][3] = {}, Fbn[3][3] = {};
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                double s1 = 0.0, s2 = 0.0;
                for (int k = 0; k < D; ++k) {
                    s1 += ((r == k ? 1.0 : 0.0) + dt * L[k][r]) * Fb[k][c];
                    s2 += Fb[r][k] * F[c][k];
                }
                Fbn[r][c] = s1;
                Lb[r][c] = dt * s2;
            }
        double xb[3] = {}, vbp[3] = {}, vpicb[3] = {}, dvb[3] = {}, Bb[3][3] = {};
        for (int d = 0; d < D; ++d) {
            xb[d] = a.x[d][i];
            vbp[d] = a.v[d][i];
            if (apic) {
                vpicb[d] = vbp[d] + dt * xb[d];
            } else {
                dvb[d] = alpha * vbp[d];
                vpicb[d] = (1.0 - alpha) * vbp[d] + dt * xb[d];
            }
        }
        if (apic)
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) Bb[r][c] = a.B[r + c * D][i];
        for_nodes(W, [&](int s, int64_t I, const int64_t* node) {
            double vi[3] = {}, vni[3] = {}, rel[3] = {};
            for (int d = 0; d < D; ++d) {
                vi[d] = double(CP<T>(g.v[d])[I]);
                vni[d] = double(CP<T>(g.vn[d])[I]);
                rel[d] = double(node_coord(M, d, node[d])) - double(x[d]);
            }
            double Nb = 0.0, Gb[3] = {0, 0, 0};
            for (int r = 0; r < D; ++r) {
                double vb_r = A.w[s] * (vpicb[r] + dvb[r]);
                for (int c = 0; c < D; ++c) vb_r += Lb[r][c] * A.g[s][c];
                Nb += vpicb[r] * vi[r] + dvb[r] * (vi[r] - vni[r]);
                for (int c = 0; c < D; ++c) Gb[c] += Lb[r][c] * vi[r];
                if (apic) {
                    double Br = 0.0;
                    for (int c = 0; c < D; ++c) {
                        Br += Bb[r][c] * rel[c];
                        xb[c] -= A.w[s] * vi[r] * Bb[r][c];  // through r = x_i - x_p
                    }
                    vb_r += A.w[s] * Br;
                    Nb += vi[r] * Br;
                }
                vb[size_t(r) * nn + I] += vb_r;
                vnb[size_t(r) * nn + I] += -A.w[s] * dvb[r];
            }
            for (int b = 0; b < D; ++b) {
                double h = 0.0;
                for (int c = 0; c < D; ++c) h += Gb[c] * A.dG[s][c][b];
                xb[b] += Nb * A.dN[s][b] + h;
            }
        });
        for (int d = 0; d < D; ++d) {
            a.x[d][i] = xb[d];
            a.v[d][i] = apic ? 0.0 : alpha * vbp[d];
        }
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                a.F[r + c * D][i] = Fbn[r][c];
                if (apic) a.B[r + c * D][i] = 0.0;
            }
    }
    // ---- grid update backwards (walled components were overwritten with 0)
    for (int64_t I = 0; I < nn; ++I) {
        const double m = double(CP<T>(g.m)[I]);
        int64_t idx[3] = {0, 0, 0}, r = I;
        for (int d = 0; d < D; ++d) { idx[d] = r % M.n[d]; r /= M.n[d]; }
        double acc = 0.0;
        for (int d = 0; d < D; ++d) {
            double v_b = vb[size_t(d) * nn + I], vn_b = vnb[size_t(d) * nn + I];
            const bool lo = (prm.wall_mask >> (2 * d)) & 1, hi = (prm.wall_mask >> (2 * d + 1)) & 1;
            if ((lo && idx[d] < prm.wall_layers) || (hi && idx[d] >= M.n[d] - prm.wall_layers)) v_b = vn_b = 0.0;
            if (m == 0.0) continue;
            const double vt = vn_b + v_b;
            fb[size_t(d) * nn + I] = dt * v_b / m;
            pb[size_t(d) * nn + I] = vt / m;
            acc += vt * double(CP<T>(g.mv[d])[I]) + dt * v_b * double(CP<T>(g.f[d])[I]);
        }
        mb[I] = (m == 0.0) ? 0.0 : -acc / (m * m);
    }
    // ---- P2G backwards
    for (int64_t i = 0; i < p.n; ++i) {
        ParticleIn<D, T> q;
        load_particle<D, T>(p, prm, i, q);
        Weights<D, T> W;
        compute_weights(M, prm.basis, q.x, q.l, W);
        double xb[3] = {}, vbs[3] = {}, sb[3][3] = {}, Vb = 0.0, Bbs[3][3] = {};
        if (!W.empty) {
            GenAdjWeights<D> A{};
            general_adjoint_weights(mraw, prm.basis, q.x, q.l, W, A);
            const double mp = double(q.m), Vp = double(q.V);
            for_nodes(W, [&](int s, int64_t I, const int64_t* node) {
                double rel[3] = {}, u[3] = {};
                for (int d = 0; d < D; ++d) rel[d] = double(node_coord(M, d, node[d])) - double(q.x[d]);
                for (int d = 0; d < D; ++d) {
                    u[d] = double(q.v[d]);
                    if (apic)
                        for (int c = 0; c < D; ++c) u[d] += double(q.B[d][c]) * dinv * rel[c];
                }
                double Nb = mp * mb[I], Gb[3] = {0, 0, 0};
                for (int d = 0; d < D; ++d) {
                    const double p_b = pb[size_t(d) * nn + I], f_b = fb[size_t(d) * nn + I];
                    Nb += mp * (u[d] * p_b + double(T(prm.gravity[d])) * f_b);
                    const double ub = mp * A.w[s] * p_b;  // d loss / d u_d
                    vbs[d] += ub;
                    if (apic)
                        for (int c = 0; c < D; ++c) {
                            Bbs[d][c] += ub * dinv * rel[c];
                            xb[c] -= ub * double(q.B[d][c]) * dinv;  // through r = x_i - x_p
                        }
                }
                for (int r = 0; r < D; ++r) {
                    const double f_b = fb[size_t(r) * nn + I];
                    double sg = 0.0;
                    for (int c = 0; c < D; ++c) {
                        sg += double(q.sig[r][c]) * A.g[s][c];
                        Gb[c] += -Vp * double(q.sig[r][c]) * f_b;
                        sb[r][c] += -Vp * f_b * A.g[s][c];
                    }
                    Vb += -f_b * sg;
                }
                for (int b = 0; b < D; ++b) {
                    double h = 0.0;
                    for (int c = 0; c < D; ++c) h += Gb[c] * A.dG[s][c][b];
                    xb[b] += Nb * A.dN[s][b] + h;
                }
            });
        }
        double F[3][3] = {}, Fb[3][3] = {}, mub = 0.0, lamb = 0.0;
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) F[r][c] = CP<double>(p.F[r + c * D])[i];
        const double mu = p.mu ? double(CP<T>(p.mu)[i]) : prm.mu;
        const double lam = p.lambda ? double(CP<T>(p.lambda)[i]) : prm.lambda;
        const double V0 = p.V0 ? double(CP<T>(p.V0)[i]) : prm.V0;
        constitutive_adjoint<D>(F, mu, lam, V0, prm.material, sb, Vb, Fb, mub, lamb);
        for (int d = 0; d < D; ++d) {
            a.x[d][i] += xb[d];
            a.v[d][i] += vbs[d];
        }
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                a.F[r + c * D][i] += Fb[r][c];
                if (apic) a.B[r + c * D][i] += Bbs[r][c];
            }
        if (a.mu) a.mu[i] += mub;
        if (a.lambda) a.lambda[i] += lamb;
    }
    return TB_OK;
}

// One step backwards on the CPU. `p` is the state at the start of the step,
// `g` receives the step's forward grid, `a` holds the sensitivities to the
// end-of-step state on entry and to the start-of-step state on return.
template <int D, class T>
inline int adjoint_step(const Mesh<D, T>& M, tb_particles& p, tb_grid& g, const tb_step_params& prm,
                        tb_adjoint& a) {
    if (!adjoint_supported(prm)) return TB_ERR_UNSUPPORTED;
    p2g<D, T>(M, p, g, prm);
    grid_update<D, T>(M, g, prm);
    const int64_t nn = M.nnodes;
    const size_t ndn = static_cast<size_t>(D) * static_cast<size_t>(nn);
    std::vector<double> vb(ndn, 0.0), vnb(ndn, 0.0), pb(ndn, 0.0), fb(ndn, 0.0);
    std::vector<double> mb(static_cast<size_t>(nn), 0.0);
    const double dt = prm.dt, alpha = prm.flip_alpha;
    // ---- G2P backwards: particle sensitivities in place, grid v / vn sensitivities scattered
    for (int64_t i = 0; i < p.n; ++i) {
        T x[3] = {0, 0, 0};
        for (int d = 0; d < D; ++d) x[d] = CP<T>(p.x[d])[i];
        const T l = opt<T>(p.l, i, prm.gimp_l);
        Weights<D, T> W;
        compute_weights(M, prm.basis, x, l, W);
        AdjWeights<D> A{};
        if (!W.empty) adjoint_weights(M, prm.basis, x, l, W, A);
        double L[3][3] = {};
        auto for_nodes = [&](auto&& fn) {
            if (W.empty) return;
            for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
                for (int j = 0; j < W.cnt[1]; ++j)
                    for (int ii = 0; ii < W.cnt[0]; ++ii) {
                        const int s = ii + 3 * j + (D == 3 ? 9 * k : 0);
                        int64_t node[3] = {W.lo[0] + ii, W.lo[1] + j, W.lo[2] + k};
                        fn(s, node_linear<D>(M.n, node));
                    }
        };
        for_nodes([&](int s, int64_t I) {
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) L[r][c] += double(CP<T>(g.v[r])[I]) * A.g[s][c];
        });
        double F[3][3] = {}, Fb[3][3] = {};
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                F[r][c] = CP<double>(p.F[r + c * D])[i];
                Fb[r][c] = a.F[r + c * D][i];
            }
        double Lb[3][3] = {}, Fbn[3][3] = {};
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                double s1 = 0.0, s2 = 0.0;
                for (int k = 0; k < D; ++k) {
                    s1 += ((r == k ? 1.0 : 0.0) + dt * L[k][r]) * Fb[k][c];  // (I + dt L)^T F_bar
                    s2 += Fb[r][k] * F[c][k];                                // F_bar F^T
                }
                Fbn[r][c] = s1;
                Lb[r][c] = dt * s2;
            }
        double xb[3] = {}, vbp[3] = {}, dvb[3] = {}, vpb[3] = {};
        for (int d = 0; d < D; ++d) {
            xb[d] = a.x[d][i];
            vbp[d] = a.v[d][i];
            dvb[d] = alpha * vbp[d];
            vpb[d] = (1.0 - alpha) * vbp[d] + dt * xb[d];
        }
        for_nodes([&](int s, int64_t I) {
            double vi[3], vni[3], gb[3] = {0, 0, 0}, wb = 0.0;
            for (int d = 0; d < D; ++d) {
                vi[d] = double(CP<T>(g.v[d])[I]);
                vni[d] = double(CP<T>(g.vn[d])[I]);
            }
            for (int r = 0; r < D; ++r) {
                double lg = 0.0;
                for (int c = 0; c < D; ++c) lg += Lb[r][c] * A.g[s][c];
                vb[size_t(r) * nn + I] += A.w[s] * (vpb[r] + dvb[r]) + lg;
                vnb[size_t(r) * nn + I] += -A.w[s] * dvb[r];
                wb += vpb[r] * vi[r] + dvb[r] * (vi[r] - vni[r]);
                for (int c = 0; c < D; ++c) gb[c] += Lb[r][c] * vi[r];
            }
            for (int b = 0; b < D; ++b) {
                double h = 0.0;
                for (int c = 0; c < D; ++c) h += A.H[s][b][c] * gb[c];
                xb[b] += wb * A.g[s][b] + h;
            }
        });
        for (int d = 0; d < D; ++d) {
            a.x[d][i] = xb[d];
            a.v[d][i] = alpha * vbp[d];
        }
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) a.F[r + c * D][i] = Fbn[r][c];
    }
    // ---- grid update backwards (walled components were overwritten with 0)
    for (int64_t I = 0; I < nn; ++I) {
        const double m = double(CP<T>(g.m)[I]);
        int64_t idx[3] = {0, 0, 0}, r = I;
        for (int d = 0; d < D; ++d) { idx[d] = r % M.n[d]; r /= M.n[d]; }
        double acc = 0.0;
        for (int d = 0; d < D; ++d) {
            double v_b = vb[size_t(d) * nn + I], vn_b = vnb[size_t(d) * nn + I];
            const bool lo = (prm.wall_mask >> (2 * d)) & 1, hi = (prm.wall_mask >> (2 * d + 1)) & 1;
            if ((lo && idx[d] < prm.wall_layers) || (hi && idx[d] >= M.n[d] - prm.wall_layers)) v_b = vn_b = 0.0;
            if (m == 0.0) continue;
            const double vt = vn_b + v_b;
            fb[size_t(d) * nn + I] = dt * v_b / m;
            pb[size_t(d) * nn + I] = vt / m;
            acc += vt * double(CP<T>(g.mv[d])[I]) + dt * v_b * double(CP<T>(g.f[d])[I]);
        }
        mb[I] = (m == 0.0) ? 0.0 : -acc / (m * m);
    }
    // ---- P2G backwards: gather into x, v and (through sigma, V) into F, mu, lambda
    for (int64_t i = 0; i < p.n; ++i) {
        ParticleIn<D, T> q;
        load_particle<D, T>(p, prm, i, q);
        Weights<D, T> W;
        compute_weights(M, prm.basis, q.x, q.l, W);
        double xb[3] = {}, vbs[3] = {}, sb[3][3] = {}, Vb = 0.0;
        if (!W.empty) {
            AdjWeights<D> A{};
            adjoint_weights(M, prm.basis, q.x, q.l, W, A);
            const double mp = double(q.m), Vp = double(q.V);
            for (int k = 0; k < (D == 3 ? W.cnt[2] : 1); ++k)
                for (int j = 0; j < W.cnt[1]; ++j)
                    for (int ii = 0; ii < W.cnt[0]; ++ii) {
                        const int s = ii + 3 * j + (D == 3 ? 9 * k : 0);
                        int64_t node[3] = {W.lo[0] + ii, W.lo[1] + j, W.lo[2] + k};
                        const int64_t I = node_linear<D>(M.n, node);
                        double wb = mp * mb[I];
                        double gb[3] = {0, 0, 0};
                        for (int d = 0; d < D; ++d) {
                            const double p_b = pb[size_t(d) * nn + I], f_b = fb[size_t(d) * nn + I];
                            wb += mp * (double(q.v[d]) * p_b + double(T(prm.gravity[d])) * f_b);
                            vbs[d] += mp * A.w[s] * p_b;
                        }
                        for (int r = 0; r < D; ++r) {
                            const double f_b = fb[size_t(r) * nn + I];
                            double sg = 0.0;
                            for (int c = 0; c < D; ++c) {
                                sg += double(q.sig[r][c]) * A.g[s][c];
                                gb[c] += -Vp * double(q.sig[r][c]) * f_b;
                                sb[r][c] += -Vp * f_b * A.g[s][c];
                            }
                            Vb += -f_b * sg;
                        }
                        for (int b = 0; b < D; ++b) {
                            double h = 0.0;
                            for (int c = 0; c < D; ++c) h += A.H[s][b][c] * gb[c];
                            xb[b] += wb * A.g[s][b] + h;
                        }
                    }
        }
        double F[3][3] = {}, Fb[3][3] = {}, mub = 0.0, lamb = 0.0;
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) F[r][c] = CP<double>(p.F[r + c * D])[i];
        const double mu = p.mu ? double(CP<T>(p.mu)[i]) : prm.mu;
        const double lam = p.lambda ? double(CP<T>(p.lambda)[i]) : prm.lambda;
        const double V0 = p.V0 ? double(CP<T>(p.V0)[i]) : prm.V0;
        constitutive_adjoint<D>(F, mu, lam, V0, prm.material, sb, Vb, Fb, mub, lamb);
        for (int d = 0; d < D; ++d) {
            a.x[d][i] += xb[d];
            a.v[d][i] += vbs[d];
        }
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) a.F[r + c * D][i] += Fb[r][c];
        if (a.mu) a.mu[i] += mub;
        if (a.lambda) a.lambda[i] += lamb;
    }
    return TB_OK;
}

// ---------------------------------------------------------------------------
// colour-phased multithreaded step (src/Parallel/region.jl:212-256 with the
// CPUBlockStrategy partition): blocks of one colour share no support node
// because the block width (4 cells) exceeds the window reach, so the blocks of
// a colour scatter in parallel without atomics.
// ---------------------------------------------------------------------------

template <int D, class T>
inline int block_colour(const Mesh<D, T>& M, int64_t b0) {
    int col = 0;
    for (int d = 0; d < D; ++d) {
        col |= int(b0 % M.nb[d] & 1) << d;
        b0 /= M.nb[d];
    }
    return col;
}

}  // namespace tbo
