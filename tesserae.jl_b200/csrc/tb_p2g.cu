// tb_p2g.cu -- block-scheduled P2G scatter of m, mv and f
// (Tesserae.jl src/Transfer/gpu.jl:139-223; equations README.md:72-74,
// test/transfer.jl:96-97 for gravity, docs/src/transfer.md:176-178 for APIC).
//
// One CTA per non-empty grid block (grid-stride over the device block list).
// The block's particles reach the (BW+3)^D-node halo tile [BW b - 1, BW b + BW + 1]
// per axis; every support window starts at one of (BW+1)^D tile positions
// ("groups"; particles of a group share their window). Two kernels share this
// schedule.
//
// p2g_pencil_kernel (B-spline, uGIMP, KernelCorrection; FLIP/PIC). Per batch of
// up to NR particles of the block (one batch for a cube3d block):
//   1. every global load of the batch is issued first; each thread finds its
//      particles' groups and ranks within them (shared counters, then a group
//      scan), and writes a record per particle at its group-sorted slot: on
//      interior blocks (no window clipped) a compact 14-word record (m_p,
//      m_p v_p, S = -V_p sigma_p, the in-window offset t; in 3D FP32 laid out
//      for packed FP32x2 arithmetic), else the full 28-word record with the
//      axis jets. Each pencil's records start 2 words further on, so the
//      pencils a warp sweeps together read distinct banks;
//   2. a lane walks a pencil of groups along x (same window start in y, z) for
//      one (y, z) row of the window and keeps the row's 3 x-nodes in registers;
//      9 rows x 3 pencils fill a warp in 3D (3 rows x 10 in 2D). Per particle
//      and row the factors wy*wz, dy*wz, wy*dz and the force rows
//      a = S[:,0] wy wz, b = S[:,1] dy wz + S[:,2] wy dz are formed once, so each
//      of the row's nodes costs w = wx wyz, m += w m_p, mv += w (m_p v_p),
//      f += dx a + wx b; after each group the x-node the window leaves for good
//      is stored to the lane's own slot of a staging array (plain stores) and
//      the row shifts one node (a register rename in the unrolled loop);
//   3. one thread per tile node sums the at most 9 staged partials that reach
//      it in FP64 and adds the node to the grid with one global atomic per
//      non-zero value (gravity, sum w m g = g sum w m, from the summed mass).
//   Interior blocks run in one launch (MODE 1), which appends every other block
//   to a list that a second launch (MODE 2, full records) then takes one block
//   per CTA; MODE 0 takes every block with full records.
//
// p2g_group_kernel (WLS weights, APIC): the same group sort and pencil sweep
// with the general per-node weight (moment inverse, APIC affine term), the
// rows' x-nodes added to an FP64 shared tile with shared atomics, and the tile
// flushed with one global atomic per non-zero node value. FP64 holds the exact
// sum of up to 2^29 FP32 terms of equal exponent, at the same 8 bytes per value
// as a (hi, lo) FP32 Kahan pair.
#include "tb_launch.cuh"

namespace tb {

namespace {

// Record layout (in T words):
//   [0] m_p  [1..3] m_p v_p
//   [4..9] S = -V sigma (symmetric; 3 used in 2D)
//   [12..17] x jets (value, derivative * h_inv) per slot, [18..23] y, [24..29] z
//   GEN: [32..34] x_p  [36..38] v_p  [40..55] moment inverse ((D+1)^2; [40] = -1
//        marks a plain kernel)  [56..64] B_p (column-major)
// The record stride is 4 (mod 32) words: the 8 lanes of a quarter warp that
// store or load 16-byte vectors of 8 consecutive records hit 8 distinct bank
// groups (a stride of 32 words would put every record in the same banks).
template <int D, bool GEN>
struct Rec {
    static constexpr int MV = 1, S = 4, AX = 12, XP = 32, VP = 36, MI = 40, BP = 56;
    static constexpr int SIZE = GEN ? 68 : (D == 3 ? 36 : 28);
};

template <class T>
struct V4 {
    T a, b, c, d;
};
template <class T>
struct V2 {
    T a, b;
};
__device__ __forceinline__ V4<float> ld4(const float* p) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V4<double> ld4(const double* p) {
    const double2 u = *reinterpret_cast<const double2*>(p), w = *reinterpret_cast<const double2*>(p + 2);
    return {u.x, u.y, w.x, w.y};
}
__device__ __forceinline__ V2<float> ld2(const float* p) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    return {v.x, v.y};
}
__device__ __forceinline__ V2<double> ld2(const double* p) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    return {v.x, v.y};
}
__device__ __forceinline__ void st4(float* p, float a, float b, float c, float d) {
    *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
__device__ __forceinline__ void st4(double* p, double a, double b, double c, double d) {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
    *reinterpret_cast<double2*>(p + 2) = make_double2(c, d);
}

// Tile bytes rounded up to 16 so the records after it are 16-byte aligned.
template <int NCTN>
__host__ __device__ constexpr size_t tile_bytes() {
    return ((sizeof(double) * NCTN + 15) / 16) * 16;
}

// 9 warps: the 25 pencils of a 3D block fill 27 (warp, pencil) slots, one task per warp.
constexpr int P2G_THREADS = 288;

template <int D, class T, int BW, bool GEN, int NR>
__global__ void __launch_bounds__(P2G_THREADS, (sizeof(T) == 4 && !GEN) ? 2 : 1) p2g_group_kernel(DMesh<D, T> M, PView<T> P, GView<T> G, Scalars<T> s,
                                                          const int* __restrict__ totals,
                                                          const int* __restrict__ blocklist,
                                                          const int* __restrict__ offsets,
                                                          const int* __restrict__ perm, int* err) {
    constexpr int NT = P2G_THREADS;
    constexpr int TS = BW + 3;
    constexpr int TN = (D == 3) ? TS * TS * TS : TS * TS;
    constexpr int NC = 1 + 2 * D;
    constexpr int G1 = BW + 1;  // window starts per axis
    constexpr int NG = (D == 3) ? G1 * G1 * G1 : G1 * G1;
    constexpr int RS = Rec<D, GEN>::SIZE;
    constexpr int NW = NT / 32;
    constexpr int NJK = (D == 3) ? 9 : 3;  // window rows
    constexpr int NSUB = 32 / NJK;         // pencils per warp: 3 (3D), 10 (2D)
    constexpr int NPENCIL = NG / G1;
    constexpr int NTASK = (NPENCIL + NSUB - 1) / NSUB;  // 9 in 3D: one per warp
    using R = Rec<D, GEN>;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* tile = reinterpret_cast<double*>(smem_raw);
    T* rec = reinterpret_cast<T*>(smem_raw + tile_bytes<NC * TN>());
    int* gcount = reinterpret_cast<int*>(rec + NR * RS);
    int* gstart = gcount + NG;
    int* pslot = gstart + NG + 1;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nactive = totals[0];
    const bool apic = s.transfer == TB_TRANSFER_APIC;
    const T dinv = T(4) / (M.h * M.h);
    const int jk = lane % NJK, sub = lane / NJK;
    const int sj = jk % 3, sk = (D == 3) ? jk / 3 : 0;

    for (int bi = blockIdx.x; bi < nactive; bi += gridDim.x) {
        const int b = blocklist[bi] - 1;
        int org[3] = {0, 0, 0};
        {
            int r = b;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                org[d] = (r % M.nb[d]) * BW - 1;
                r /= M.nb[d];
            }
        }
        for (int t = tid; t < NC * TN; t += NT) tile[t] = 0.0;
        const int s0 = offsets[b], s1 = offsets[b + 1];
        for (int b0 = s0; b0 < s1; b0 += NR) {
            const int nbat = min(NR, s1 - b0);
            for (int g = tid; g < NG; g += NT) gcount[g] = 0;
            __syncthreads();
            // ---- 1a. group (window start) and rank of every particle of the batch
            constexpr int ITEMS = (NR + NT - 1) / NT;
            int grp[ITEMS], rank[ITEMS];
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                const int ti = tid + u * NT;
                grp[u] = -1;
                rank[u] = 0;
                if (ti >= nbat) continue;
                const long long p = perm[b0 + ti] - 1;
                T x[3];
#pragma unroll
                for (int d = 0; d < D; ++d) x[d] = P.x[d][p];
                const T l = P.l ? P.l[p] : s.gimp_l;
                Basis<D, T> B;
                if (!prepare_basis<D, T, false>(M, s.basis == TB_WLS_UGIMP ? TB_UGIMP
                                                   : (s.basis == TB_WLS_BSPLINE_QUADRATIC ? TB_BSPLINE_QUADRATIC
                                                                                           : s.basis),
                                                x, l, B, err))
                    continue;
                int gi = 0;
                bool ok = true;
#pragma unroll
                for (int d = D - 1; d >= 0; --d) {
                    const int q = B.ax[d].lo - org[d];
                    ok = ok && q >= 0 && q < G1;
                    gi = gi * G1 + q;
                }
                if (!ok) {
                    atomicOr(err, ERR_TILE_RANGE);
                    continue;
                }
                grp[u] = gi;
                rank[u] = atomicAdd(&gcount[gi], 1);
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
            } else if (warp == 1) {
                // Pencil slots by size, largest first, so the NSUB pencils a warp
                // sweeps in lockstep have similar lengths.
                int myp = lane < NPENCIL ? lane : -1;
                int mysize = 0;
                if (myp >= 0) {
                    const int gb = G1 * myp;
                    for (int gx = 0; gx < G1; ++gx) mysize += gcount[gb + gx];
                }
                int rk = 0;
                for (int o = 0; o < NPENCIL; ++o) {
                    const int os = __shfl_sync(0xffffffffu, mysize, o);
                    rk += (os > mysize) || (os == mysize && o < lane);
                }
                if (myp >= 0) pslot[rk] = myp;
            }
            __syncthreads();
            // ---- 1b. records, written at their group-sorted position
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                if (grp[u] < 0) continue;
                const int ti = tid + u * NT;
                const long long p = perm[b0 + ti] - 1;
                T x[3];
#pragma unroll
                for (int d = 0; d < D; ++d) x[d] = P.x[d][p];
                const T l = P.l ? P.l[p] : s.gimp_l;
                Basis<D, T> B;
                prepare_basis<D, T, GEN>(M, s.basis, x, l, B, err);
                T* r = rec + (gstart[grp[u]] + rank[u]) * RS;
                const T mp = P.m ? P.m[p] : s.mass;
                const T Vp = P.V[p];
                T v[3] = {T(0), T(0), T(0)};
#pragma unroll
                for (int d = 0; d < D; ++d) v[d] = P.v[d][p];
                T Sv[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) Sv[k] = (k < (D == 3 ? 6 : 3)) ? (-Vp) * P.sig[k < 6 ? k : 0][p] : T(0);
                T ax[18];
#pragma unroll
                for (int d = 0; d < 3; ++d)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        ax[6 * d + 2 * k] = d < D ? B.ax[d < D ? d : 0].val[k] : T(0);
                        ax[6 * d + 2 * k + 1] = d < D ? B.ax[d < D ? d : 0].der[k] * M.h_inv : T(0);
                    }
                st4(r + 0, mp, mp * v[0], mp * v[1], mp * v[2]);
                st4(r + 4, Sv[0], Sv[1], Sv[2], Sv[3]);
                st4(r + 8, Sv[4], Sv[5], T(0), T(0));
                st4(r + 12, ax[0], ax[1], ax[2], ax[3]);
                st4(r + 16, ax[4], ax[5], ax[6], ax[7]);
                st4(r + 20, ax[8], ax[9], ax[10], ax[11]);
                if constexpr (D == 3) {
                    st4(r + 24, ax[12], ax[13], ax[14], ax[15]);
                    st4(r + 28, ax[16], ax[17], T(0), T(0));
                }
                if constexpr (GEN) {
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        r[R::XP + d] = d < D ? x[d] : T(0);
                        r[R::VP + d] = v[d];
                    }
#pragma unroll
                    for (int i = 0; i < D + 1; ++i)
#pragma unroll
                        for (int j = 0; j < D + 1; ++j)
                            r[R::MI + i * (D + 1) + j] = B.wls ? B.Mi[i][j] : T(i == j ? 1 : 0);
                    r[R::MI] = B.wls ? B.Mi[0][0] : T(-1);
#pragma unroll
                    for (int k = 0; k < D * D; ++k) r[R::BP + k] = apic ? P.B[k][p] : T(0);
                }
            }
            __syncthreads();
            // ---- 2./3. pencils of groups along x: the NSUB lane sets of a warp
            //      walk NSUB different pencils, so every lane owns its (pencil, row)
            //      and adds its sums to the tile without any cross-lane reduction.
            for (int task = warp; task < NTASK; task += NW) {
                const int slot = task * NSUB + sub;
                const bool live = sub < NSUB && slot < NPENCIL;
                const int pc = live ? pslot[slot] : 0;
                const int gy = live ? pc % G1 : 0, gz = (D == 3 && live) ? pc / G1 : 0;
                const int gbase = G1 * (gy + G1 * gz);
                T acc[3][NC];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int c = 0; c < NC; ++c) acc[i][c] = T(0);
                T Y = T(0), Z = T(0);
                if constexpr (GEN) {
                    Y = node_coord(M, 1, org[1] + gy + sj);
                    if constexpr (D == 3) Z = node_coord(M, 2, org[2] + gz + sk);
                }
#pragma unroll
                for (int gx = 0; gx < G1 + 2; ++gx) {
                    if (gx < G1 && live) {
                        const int q1 = gstart[gbase + gx + 1];
                        for (int q = gstart[gbase + gx]; q < q1; ++q) {
                            const T* r = rec + q * RS;
                            const V4<T> m4 = ld4(r + 0), s4 = ld4(r + 4), x4 = ld4(r + 12);
                            const V2<T> s2 = ld2(r + 8), x2 = ld2(r + 16), y2 = ld2(r + R::AX + 6 + 2 * sj);
                            const T mp = m4.a;
                            const T mv[3] = {m4.b, m4.c, m4.d};
                            const T S[6] = {s4.a, s4.b, s4.c, s4.d, s2.a, s2.b};
                            const T wx[3] = {x4.a, x4.c, x2.a}, dx[3] = {x4.b, x4.d, x2.b};
                            const T wy = y2.a, dy = y2.b;
                            T wyz, dyz, wdz;
                            if constexpr (D == 3) {
                                const V2<T> z2 = ld2(r + R::AX + 12 + 2 * sk);
                                const T wz = z2.a, dz = z2.b;
                                wyz = wy * wz;
                                dyz = dy * wz;
                                wdz = wy * dz;
                            } else {
                                wyz = wy;
                                dyz = dy;
                                wdz = T(0);
                            }
                            if constexpr (!GEN) {
                                // f_a = S[a,0] dx wyz + S[a,1] wx dyz + S[a,2] wx wdz
                                T fa[3], fb[3];
#pragma unroll
                                for (int a = 0; a < D; ++a) {
                                    fa[a] = S[symidx<D>(a, 0)] * wyz;
                                    fb[a] = S[symidx<D>(a, 1)] * dyz;
                                    if constexpr (D == 3) fb[a] += S[symidx<D>(a, 2)] * wdz;
                                }
#pragma unroll
                                for (int i = 0; i < 3; ++i) {
                                    const T w = wx[i] * wyz;
                                    acc[i][0] += w * mp;
#pragma unroll
                                    for (int d = 0; d < D; ++d) acc[i][1 + d] += w * mv[d];
#pragma unroll
                                    for (int a = 0; a < D; ++a) acc[i][1 + D + a] += dx[i] * fa[a] + wx[i] * fb[a];
                                }
                            } else {
#pragma unroll
                                for (int i = 0; i < 3; ++i) {
                                    T w = wx[i] * wyz;
                                    T gw[3] = {dx[i] * wyz, wx[i] * dyz, wx[i] * wdz};
                                    T rel[3];
                                    rel[0] = node_coord(M, 0, org[0] + gx + i) - r[R::XP + 0];
                                    rel[1] = Y - r[R::XP + 1];
                                    rel[2] = (D == 3) ? Z - r[R::XP + 2] : T(0);
                                    if (r[R::MI] != T(-1)) {  // WLS: wq = w Mi [1; rel]
                                        constexpr int N = D + 1;
                                        T Pv[N];
                                        Pv[0] = T(1);
#pragma unroll
                                        for (int d = 0; d < D; ++d) Pv[d + 1] = rel[d];
                                        T wq[N];
#pragma unroll
                                        for (int a = 0; a < N; ++a) {
                                            T t = T(0);
#pragma unroll
                                            for (int c = 0; c < N; ++c) t += r[R::MI + a * N + c] * Pv[c];
                                            wq[a] = w * t;
                                        }
                                        w = wq[0];
#pragma unroll
                                        for (int d = 0; d < D; ++d) gw[d] = wq[d + 1];
                                    }
                                    T vv[3];
#pragma unroll
                                    for (int d = 0; d < D; ++d) vv[d] = r[R::VP + d];
                                    if (apic) {
#pragma unroll
                                        for (int a = 0; a < D; ++a) {
                                            T t = T(0);
#pragma unroll
                                            for (int c = 0; c < D; ++c) t += r[R::BP + a + c * D] * dinv * rel[c];
                                            vv[a] += t;
                                        }
                                    }
                                    const T wm = w * mp;
                                    acc[i][0] += wm;
#pragma unroll
                                    for (int d = 0; d < D; ++d) acc[i][1 + d] += wm * vv[d];
#pragma unroll
                                    for (int a = 0; a < D; ++a) {
                                        T t = S[symidx<D>(a, 0)] * gw[0];
#pragma unroll
                                        for (int c = 1; c < D; ++c) t += S[symidx<D>(a, c)] * gw[c];
                                        acc[i][1 + D + a] += t;
                                    }
                                }
                            }
                        }
                    }
                    // Column gx (slot 0) is final: later groups start further right.
                    if (live && gx < TS) {
                        const int tj = gy + sj, tk = (D == 3) ? gz + sk : 0;
                        const int t = (D == 3) ? gx + TS * (tj + TS * tk) : gx + TS * tj;
#pragma unroll
                        for (int c = 0; c < NC; ++c)
                            if (acc[0][c] != T(0)) atomicAdd(&tile[c * TN + t], double(acc[0][c]));
                    }
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        acc[0][c] = acc[1][c];
                        acc[1][c] = acc[2][c];
                        acc[2][c] = T(0);
                    }
                }
            }
            __syncthreads();
        }
        // ---- flush the tile
        for (int t = tid; t < TN; t += NT) {
            int node[3] = {0, 0, 0}, rem = t;
            bool inside = true;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                node[d] = org[d] + rem % TS;
                rem /= TS;
                inside = inside && node[d] >= 0 && node[d] < M.n[d];
            }
            if (!inside) continue;
            double val[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) val[c] = tile[c * TN + t];
#pragma unroll
            for (int d = 0; d < D; ++d) val[1 + D + d] += double(s.g[d]) * val[0];
            grid_add<D>(G, M, err, node[0], node[1], D == 3 ? node[2] : 0, val);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Plain kernel (B-spline or uGIMP, FLIP/PIC blend): the same pencil sweep
// without shared-memory atomics.
//   1a. window start only (no basis values) -> group and rank in the group;
//   1b. basis jets once per particle, record written at its group-sorted slot;
//   2.  a lane walks its pencil's groups in x order, two records in flight at a
//       time; after each group the x-node the window leaves for good is final
//       for this (pencil, row) and is stored, with plain stores, to the lane's
//       own slot of a staging array (the group loop is unrolled, so the shift of
//       the 3-node row is a register rename);
//   3.  one thread per tile node sums the at most 3^(D-1) staged partials that
//       reach it (pencils gy = ty - sj, gz = tz - sk) in FP64 and adds the node
//       to the grid with one global atomic per non-zero value.
// On B200 an FP64 shared-memory atomic add is a compare-and-swap loop; in the
// tiled form of this sweep those atomics retried 2.5 times each and, with the
// record loads, kept the shared-memory pipe at 69% of its wavefront rate. The
// staged form issues no shared atomic. Partials are the FP32 sums of one
// pencil row (at most 3 groups); the sum over pencils is FP64.
//
// Record (T words): [0] m_p [1..3] m_p v_p [4..9] S = -V_p sigma_p (Tensorial
// symmetric order; 3 used in 2D) [10..15] x jets (value, h_inv-scaled
// derivative per slot) [16..21] y jets [22..27] z jets. 28 words = 7 x 16 bytes,
// so 8 consecutive records stored as 16-byte vectors hit 8 distinct bank groups.
constexpr int PRS = 28;

__device__ __forceinline__ void st2(float* p, float a, float b) { *reinterpret_cast<float2*>(p) = make_float2(a, b); }
__device__ __forceinline__ void st2(double* p, double a, double b) {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
}

template <class T>
struct PlainRec {
    V4<T> m4, s4, xb;
    V2<T> s2, xa, y2, z2;
};

template <int D, class T>
__device__ __forceinline__ void load_plain(const T* r, int sj, int sk, PlainRec<T>& o) {
    o.m4 = ld4(r + 0);
    o.s4 = ld4(r + 4);
    if constexpr (D == 3) o.s2 = ld2(r + 8);
    o.xa = ld2(r + 10);
    o.xb = ld4(r + 12);
    o.y2 = ld2(r + 16 + 2 * sj);
    if constexpr (D == 3) o.z2 = ld2(r + 22 + 2 * sk);
}

template <int D, class T>
__device__ __forceinline__ void accumulate_plain(const PlainRec<T>& o, T (&acc)[3][1 + 2 * D]) {
    const T mp = o.m4.a;
    const T mv[3] = {o.m4.b, o.m4.c, o.m4.d};
    T S[6] = {o.s4.a, o.s4.b, o.s4.c, o.s4.d, T(0), T(0)};
    if constexpr (D == 3) {
        S[4] = o.s2.a;
        S[5] = o.s2.b;
    }
    const T wx[3] = {o.xa.a, o.xb.a, o.xb.c}, dx[3] = {o.xa.b, o.xb.b, o.xb.d};
    T wyz, dyz, wdz = T(0);
    if constexpr (D == 3) {
        wyz = o.y2.a * o.z2.a;
        dyz = o.y2.b * o.z2.a;
        wdz = o.y2.a * o.z2.b;
    } else {
        wyz = o.y2.a;
        dyz = o.y2.b;
    }
    // f_a = S[a,0] dx wyz + S[a,1] wx dyz + S[a,2] wx wdz
    T fa[3], fb[3];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        fa[a] = S[symidx<D>(a, 0)] * wyz;
        fb[a] = S[symidx<D>(a, 1)] * dyz;
        if constexpr (D == 3) fb[a] += S[symidx<D>(a, 2)] * wdz;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T w = wx[i] * wyz;
        acc[i][0] += w * mp;
#pragma unroll
        for (int d = 0; d < D; ++d) acc[i][1 + d] += w * mv[d];
#pragma unroll
        for (int a = 0; a < D; ++a) acc[i][1 + D + a] += dx[i] * fa[a] + wx[i] * fb[a];
    }
}

// Compact record (interior blocks of a quadratic B-spline, where no window is
// truncated): [0] m_p [1..3] m_p v_p [4..9] S [10..12] t per axis, the fast
// path's t = fract(xi - 1/2) (bspline.jl:90-100), [13] unused. 14 words: the
// row lanes evaluate the 1-D jets from t with the polynomial of
// bspline_quadratic_poly, so the weights agree with the full record's to
// rounding. Records are 8-byte aligned (56-byte stride).
constexpr int CRS = 14;

// Coefficients of the quadratic B-spline slot k as a + t (b + t c) and its
// derivative e + t f (bspline_quadratic_poly, slot by slot).
struct SlotPoly {
    float a, b, c, e, f;
};
__device__ __forceinline__ SlotPoly slot_poly(int k) {
    if (k == 0) return {0.5f, -1.0f, 0.5f, -1.0f, 1.0f};
    if (k == 1) return {0.5f, 1.0f, -1.0f, 1.0f, -2.0f};
    return {0.0f, 0.0f, 0.5f, 0.0f, 1.0f};
}

template <class T>
struct CompactRec {
    V2<T> m0, m1, s0, s1, s2, t01, t2;
};

template <int D, class T>
__device__ __forceinline__ void load_compact(const T* r, CompactRec<T>& o) {
    o.m0 = ld2(r + 0);
    o.m1 = ld2(r + 2);
    o.s0 = ld2(r + 4);
    o.s1 = ld2(r + 6);
    if constexpr (D == 3) o.s2 = ld2(r + 8);
    o.t01 = ld2(r + 10);
    if constexpr (D == 3) o.t2 = ld2(r + 12);
}

template <int D, class T>
__device__ __forceinline__ void accumulate_compact(const CompactRec<T>& o, const SlotPoly& py, const SlotPoly& pz,
                                                   T h_inv, T (&acc)[3][1 + 2 * D]) {
    const T mp = o.m0.a;
    const T mv[3] = {o.m0.b, o.m1.a, o.m1.b};
    T S[6] = {o.s0.a, o.s0.b, o.s1.a, o.s1.b, T(0), T(0)};
    if constexpr (D == 3) {
        S[4] = o.s2.a;
        S[5] = o.s2.b;
    }
    const T tx = o.t01.a, ty = o.t01.b;
    const T half = T(0.5);
    const T wx[3] = {half + tx * (T(-1) + tx * half), half + tx * (T(1) + tx * T(-1)), tx * (tx * half)};
    const T dx[3] = {(T(-1) + tx) * h_inv, (T(1) + tx * T(-2)) * h_inv, tx * h_inv};
    const T wy = T(py.a) + ty * (T(py.b) + ty * T(py.c));
    const T dy = (T(py.e) + ty * T(py.f)) * h_inv;
    T wyz, dyz, wdz = T(0);
    if constexpr (D == 3) {
        const T tz = o.t2.a;
        const T wz = T(pz.a) + tz * (T(pz.b) + tz * T(pz.c));
        const T dz = (T(pz.e) + tz * T(pz.f)) * h_inv;
        wyz = wy * wz;
        dyz = dy * wz;
        wdz = wy * dz;
    } else {
        wyz = wy;
        dyz = dy;
    }
    T fa[3], fb[3];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        fa[a] = S[symidx<D>(a, 0)] * wyz;
        fb[a] = S[symidx<D>(a, 1)] * dyz;
        if constexpr (D == 3) fb[a] += S[symidx<D>(a, 2)] * wdz;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T w = wx[i] * wyz;
        acc[i][0] += w * mp;
#pragma unroll
        for (int d = 0; d < D; ++d) acc[i][1 + d] += w * mv[d];
#pragma unroll
        for (int a = 0; a < D; ++a) acc[i][1 + D + a] += dx[i] * fa[a] + wx[i] * fb[a];
    }
}

// 3D FP32 compact record, laid out for packed FP32x2 arithmetic (S = -V sigma in
// Tensorial order 11 21 31 22 32 33 = S0..S5):
//   (m, m v_x) (m v_y, m v_z) (S0, S1) (S1, S3) (S2, S4) (S5, t_z) (t_x, t_y)
// so that f_xy = dx (S0, S1) wyz + wx ((S1, S3) dyz + (S2, S4) wdz) is pairwise.
struct PairRec {
    float2 m0, m1, sa, sb, sc, s5z, txy;
};
__device__ __forceinline__ void load_pair_rec(const float* r, PairRec& o) {
    o.m0 = *reinterpret_cast<const float2*>(r + 0);
    o.m1 = *reinterpret_cast<const float2*>(r + 2);
    o.sa = *reinterpret_cast<const float2*>(r + 4);
    o.sb = *reinterpret_cast<const float2*>(r + 6);
    o.sc = *reinterpret_cast<const float2*>(r + 8);
    o.s5z = *reinterpret_cast<const float2*>(r + 10);
    o.txy = *reinterpret_cast<const float2*>(r + 12);
}
// Per x-node of a row lane: (m, m v_x), (m v_y, m v_z), (f_x, f_y) and f_z.
struct PairAcc {
    float2 a01, a23, f01;
    float f2;
};
__device__ __forceinline__ void accumulate_pair(const PairRec& o, const SlotPoly& py, const SlotPoly& pz, float h_inv,
                                                PairAcc (&acc)[3]) {
    const float tx = o.txy.x, ty = o.txy.y, tz = o.s5z.y;
    const float2 t2 = make_float2(tx, tx);
    // (wx_i, wx_i) and (dx_i, dx_i): the B-spline factors of the three x slots
    const float2 wx0 = __ffma2_rn(t2, __ffma2_rn(t2, make_float2(0.5f, 0.5f), make_float2(-1.f, -1.f)),
                                  make_float2(0.5f, 0.5f));
    const float2 wx1 = __ffma2_rn(t2, __ffma2_rn(t2, make_float2(-1.f, -1.f), make_float2(1.f, 1.f)),
                                  make_float2(0.5f, 0.5f));
    const float2 wx2 = __fmul2_rn(t2, __fmul2_rn(t2, make_float2(0.5f, 0.5f)));
    const float2 hh = make_float2(h_inv, h_inv);
    const float2 dx0 = __fmul2_rn(__fadd2_rn(t2, make_float2(-1.f, -1.f)), hh);
    const float2 dx1 = __fmul2_rn(__ffma2_rn(t2, make_float2(-2.f, -2.f), make_float2(1.f, 1.f)), hh);
    const float2 dx2 = __fmul2_rn(t2, hh);
    const float wy = py.a + ty * (py.b + ty * py.c);
    const float dy = (py.e + ty * py.f) * h_inv;
    const float wz = pz.a + tz * (pz.b + tz * pz.c);
    const float dz = (pz.e + tz * pz.f) * h_inv;
    const float wyz = wy * wz, dyz = dy * wz, wdz = wy * dz;
    const float2 WYZ = make_float2(wyz, wyz);
    const float2 fa01 = __fmul2_rn(o.sa, WYZ);
    const float2 fb01 = __ffma2_rn(o.sc, make_float2(wdz, wdz), __fmul2_rn(o.sb, make_float2(dyz, dyz)));
    const float fa2 = o.sc.x * wyz;
    const float fb2 = __fmaf_rn(o.s5z.x, wdz, o.sc.y * dyz);
    const float2 wxs[3] = {wx0, wx1, wx2}, dxs[3] = {dx0, dx1, dx2};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float2 w = __fmul2_rn(wxs[i], WYZ);
        acc[i].a01 = __ffma2_rn(w, o.m0, acc[i].a01);
        acc[i].a23 = __ffma2_rn(w, o.m1, acc[i].a23);
        acc[i].f01 = __ffma2_rn(dxs[i], fa01, __ffma2_rn(wxs[i], fb01, acc[i].f01));
        acc[i].f2 = __fmaf_rn(dxs[i].x, fa2, __fmaf_rn(wxs[i].x, fb2, acc[i].f2));
    }
}

template <int NC, class T>
__device__ __forceinline__ void stage_node(T* part, int base, int stride, const T (&a)[NC]) {
#pragma unroll
    for (int c = 0; c < NC; ++c) part[base + c * stride] = a[c];
}

// Staging layout: partial (component c, row jk, pencil pc, tile x) at
// ((c * NJK + jk) * NPENCIL + pc) * TS + x. For one row offset jk the pencils
// (gy, gz) of a tile plane follow each other, so the gather's reads for
// consecutive tile nodes are consecutive words (no bank conflicts within a
// plane).
template <int D, int BW>
struct PencilShape {
    static constexpr int TS = BW + 3;
    static constexpr int TN = (D == 3) ? TS * TS * TS : TS * TS;
    static constexpr int NC = 1 + 2 * D;
    static constexpr int G1 = BW + 1;
    static constexpr int NG = (D == 3) ? G1 * G1 * G1 : G1 * G1;
    static constexpr int NJK = (D == 3) ? 9 : 3;
    static constexpr int NSUB = 32 / NJK;
    static constexpr int NPENCIL = NG / G1;
    static constexpr int NPART = NC * NPENCIL * NJK * TS;
    // Records of pencil pc start skew * pc words after their slot: pencils of
    // equal size (multiples of 8 records on a regular lattice) would otherwise
    // put the records a warp's three pencils read together in the same banks.
    // 2 words keeps 8-byte records loads aligned, 4 the 16-byte ones of FP32
    // full records.
    static constexpr int skew(int mode, int tsize) { return (mode == 1 || tsize == 8) ? 2 : 4; }
};

// MODE 0: every block with the full record; 1: compact records, interior
// blocks only (their halo tile lies inside the mesh, so no window is
// truncated), appending every other block it meets to `bnd` (count in
// `bnd_count`, zeroed before); 2: full records, the blocks of that list, one
// per CTA at a time (the boundary blocks of a scene can all sit in one stretch
// of the block list, e.g. a body standing on the mesh floor).
template <int D, class T, int BW, int NR, bool X64, int MODE>
__global__ void __launch_bounds__(P2G_THREADS, MODE == 1 ? 3 : (sizeof(T) == 4 ? 2 : 1)) p2g_pencil_kernel(DMesh<D, T> M, PView<T> P, GView<T> G, Scalars<T> s,
                                                                    const int* __restrict__ totals,
                                                                    const int* __restrict__ blocklist,
                                                                    const int* __restrict__ offsets,
                                                                    const int* __restrict__ perm, int* err,
                                                                    int* __restrict__ bnd,
                                                                    unsigned long long* __restrict__ bnd_count) {
    using SH = PencilShape<D, BW>;
    constexpr int NT = P2G_THREADS;
    constexpr int TS = SH::TS, TN = SH::TN, NC = SH::NC, G1 = SH::G1, NG = SH::NG;
    constexpr int NW = NT / 32;
    constexpr int NJK = SH::NJK, NSUB = SH::NSUB, NPENCIL = SH::NPENCIL;
    constexpr int NTASK = (NPENCIL + NSUB - 1) / NSUB;
    constexpr int ITEMS = (NR + NT - 1) / NT;
    constexpr int CSTR = NPENCIL * NJK * TS;  // stride between components in the staging array
    static_assert(NPENCIL <= 32, "pencil ranking runs in one warp");
    static_assert(NR % 8 == 0 && NT % 8 == 0, "passes in 8-particle chunks");

    constexpr int RS = (MODE == 1) ? CRS : PRS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int SKW = SH::skew(MODE, sizeof(T));
    // 3D FP32 compact records: packed FP32x2 accumulation (PairRec layout)
    constexpr bool PAIRS = (MODE == 1 && D == 3 && sizeof(T) == 4);
    T* rec = reinterpret_cast<T*>(smem_raw);
    T* part = rec + NR * RS + SKW * NPENCIL;
    int* gcount = reinterpret_cast<int*>(part + SH::NPART);
    int* gstart = gcount + NG;
    int* pslot = gstart + NG + 1;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nactive = totals[0];
    const int jk = lane % NJK, sub = lane / NJK;
    const int sj = jk % 3, sk = (D == 3) ? jk / 3 : 0;
    const bool gimp = basis_is_gimp(s.basis);
    const SlotPoly py = slot_poly(sj), pz = slot_poly(sk);

    for (int g = tid; g < NG; g += NT) gcount[g] = 0;
    __syncthreads();

    // interior block: its halo tile lies inside the mesh, so no window is truncated
    auto interior_block = [&](int b) {
        bool in = true;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const int o = (b % M.nb[d]) * BW - 1;
            b /= M.nb[d];
            in = in && o >= 0 && o + TS - 1 <= M.n[d] - 1;
        }
        return in;
    };
    auto process_block = [&](const int b, const int piece, const int pieces) {
        int org[3] = {0, 0, 0};
        {
            int r = b;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                org[d] = (r % M.nb[d]) * BW - 1;
                r /= M.nb[d];
            }
        }
        const int s0 = offsets[b], s1 = offsets[b + 1];
        const BlockPasses bp(s0, s1, NR);
        for (int bi = piece; bi < bp.count(); bi += pieces) {
            const int q0 = bp.pos(bi, tid), qstep = bp.step(NT);
            // ---- 1a. every global load of the batch first (the ids, then all of
            //      the particles' fields at once: two dependent round trips per
            //      batch), then window start -> group, rank within the group. The
            //      fields stay in registers for 1b.
            int grp[ITEMS], rank[ITEMS];
            long long pid[ITEMS];
            T px[ITEMS][3], pv[ITEMS][3], pV[ITEMS], pm[ITEMS], pl[ITEMS], psg[ITEMS][6];
            double pxd[ITEMS][3];
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                const int ti = tid + u * NT, q = q0 + u * qstep;
                pid[u] = (ti < NR && q < s1) ? perm[q] - 1 : -1;
            }
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                const long long p = pid[u] >= 0 ? pid[u] : 0;
                const bool on = pid[u] >= 0;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if constexpr (X64) {
                        pxd[u][d] = (on && d < D) ? P.x64[d < D ? d : 0][p] : 0.0;
                        px[u][d] = T(0);
                    } else {
                        px[u][d] = (on && d < D) ? P.x[d < D ? d : 0][p] : T(0);
                        pxd[u][d] = 0.0;
                    }
                    pv[u][d] = (on && d < D) ? P.v[d < D ? d : 0][p] : T(0);
                }
                pV[u] = on ? P.V[p] : T(0);
                pm[u] = (on && P.m) ? P.m[p] : s.mass;
                pl[u] = (on && P.l) ? P.l[p] : s.gimp_l;
#pragma unroll
                for (int k = 0; k < 6; ++k) psg[u][k] = (on && k < nsym<D>()) ? P.sig[k < nsym<D>() ? k : 0][p] : T(0);
            }
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                grp[u] = -1;
                rank[u] = 0;
                if (pid[u] < 0) continue;
                int lo[3], cnt[3];
                bool inside;
                if constexpr (X64) {
                    double xi[3], lnorm = 0.0;
                    if (gimp) {
                        lnorm = double(pl[u]) / M.h64;
                        if (!(lnorm >= 0.0 && lnorm <= 1.0)) {
                            atomicOr(err, ERR_GIMP_LENGTH);
                            continue;
                        }
                    }
                    inside = axis_window_x64<D, T>(M, s.basis, pxd[u], lnorm, xi, lo, cnt);
                } else {
                    T xi[3], lnorm = T(0);
                    if (gimp) {
                        lnorm = pl[u] / M.h;
                        if (!(lnorm >= T(0) && lnorm <= T(1))) {
                            atomicOr(err, ERR_GIMP_LENGTH);
                            continue;
                        }
                    }
                    inside = axis_window<D, T>(M, s.basis, px[u], lnorm, xi, lo, cnt);
                }
                if (!inside) continue;
                int gi = 0;
                bool ok = true;
#pragma unroll
                for (int d = D - 1; d >= 0; --d) {
                    const int q = lo[d] - org[d];
                    ok = ok && q >= 0 && q < G1;
                    gi = gi * G1 + q;
                }
                if (!ok) {
                    atomicOr(err, ERR_TILE_RANGE);
                    continue;
                }
                grp[u] = gi;
                rank[u] = atomicAdd(&gcount[gi], 1);
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
            } else if (warp == 1) {
                // pencil slots by size, largest first: the NSUB pencils a warp
                // sweeps in lockstep then have similar lengths
                const int myp = lane < NPENCIL ? lane : -1;
                int mysize = 0;
                if (myp >= 0) {
                    const int gb = G1 * myp;
                    for (int gx = 0; gx < G1; ++gx) mysize += gcount[gb + gx];
                }
                int rk = 0;
                for (int o = 0; o < NPENCIL; ++o) {
                    const int os = __shfl_sync(0xffffffffu, mysize, o);
                    rk += (os > mysize) || (os == mysize && o < lane);
                }
                if (myp >= 0) pslot[rk] = myp;
            }
            __syncthreads();
            // ---- 1b. basis jets and record at the group-sorted slot
            for (int g = tid; g < NG; g += NT) gcount[g] = 0;  // ready for the next batch
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                if (grp[u] < 0) continue;
                if constexpr (MODE == 1) {
                    // t = fract(xi - 1/2) per axis, as the fast path computes it
                    T t[3] = {T(0), T(0), T(0)};
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        if constexpr (X64) {
                            const double xi = (pxd[u][d] - M.xmin64[d]) * M.h_inv64;
                            const double u64 = xi - 0.5;
                            T tt = T(u64 - floor(u64));
                            if (tt >= T(1)) tt = T(1) - T(1) / T(1 << 24);
                            t[d] = tt;
                        } else {
                            const T uu = (px[u][d] - M.xmin[d]) * M.h_inv - T(0.5);
                            t[d] = uu - floor(uu);
                        }
                    }
                    T* r = rec + (gstart[grp[u]] + rank[u]) * CRS + SKW * (grp[u] / G1);
                    const T mp = pm[u];
                    const T nV = -pV[u];
                    if constexpr (PAIRS) {
                        st2(r + 0, mp, mp * pv[u][0]);
                        st2(r + 2, mp * pv[u][1], mp * pv[u][2]);
                        st2(r + 4, nV * psg[u][0], nV * psg[u][1]);
                        st2(r + 6, nV * psg[u][1], nV * psg[u][3]);
                        st2(r + 8, nV * psg[u][2], nV * psg[u][4]);
                        st2(r + 10, nV * psg[u][5], t[2]);
                        st2(r + 12, t[0], t[1]);
                        continue;
                    }
                    st2(r + 0, mp, mp * pv[u][0]);
                    st2(r + 2, mp * pv[u][1], mp * pv[u][2]);
                    st2(r + 4, nV * psg[u][0], nV * psg[u][1]);
                    st2(r + 6, nV * psg[u][2], nV * psg[u][3]);
                    st2(r + 8, nV * psg[u][4], nV * psg[u][5]);
                    st2(r + 10, t[0], t[1]);
                    st2(r + 12, t[2], T(0));
                    continue;
                }
                Basis<D, T> B;
                if constexpr (X64) prepare_basis_x64<D, T>(M, s.basis, pxd[u], pl[u], B, err);
                else prepare_basis<D, T, false>(M, s.basis, px[u], pl[u], B, err);
                T* r = rec + (gstart[grp[u]] + rank[u]) * PRS + SKW * (grp[u] / G1);
                const T mp = pm[u];
                const T nV = -pV[u];
                const T* v = pv[u];
                T Sv[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) Sv[k] = nV * psg[u][k];
                T jv[3][3], jd[3][3];
#pragma unroll
                for (int d = 0; d < 3; ++d)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        jv[d][k] = d < D ? B.ax[d < D ? d : 0].val[k] : T(0);
                        jd[d][k] = d < D ? B.ax[d < D ? d : 0].der[k] * M.h_inv : T(0);
                    }
                st4(r + 0, mp, mp * v[0], mp * v[1], mp * v[2]);
                st4(r + 4, Sv[0], Sv[1], Sv[2], Sv[3]);
                st2(r + 8, Sv[4], Sv[5]);
                st2(r + 10, jv[0][0], jd[0][0]);
                st4(r + 12, jv[0][1], jd[0][1], jv[0][2], jd[0][2]);
                st4(r + 16, jv[1][0], jd[1][0], jv[1][1], jd[1][1]);
                st2(r + 20, jv[1][2], jd[1][2]);
                st2(r + 22, jv[2][0], jd[2][0]);
                st4(r + 24, jv[2][1], jd[2][1], jv[2][2], jd[2][2]);
            }
            __syncthreads();
            // ---- 2. pencil sweeps; every live (pencil, row) stages all TS x-nodes
            for (int task = warp; task < NTASK; task += NW) {
                const int slot = task * NSUB + sub;
                if (sub >= NSUB || slot >= NPENCIL) continue;
                const int pc = pslot[slot];
                const int gbase = G1 * pc;
                const int pbase = (jk * NPENCIL + pc) * TS;
                const T* prec = rec + SKW * pc;  // this pencil's records (skewed)
                if constexpr (PAIRS) {
                    PairAcc pa[3];
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        pa[i].a01 = pa[i].a23 = pa[i].f01 = make_float2(0.f, 0.f);
                        pa[i].f2 = 0.f;
                    }
                    const float* frec = reinterpret_cast<const float*>(prec);
                    int qs = gstart[gbase];
#pragma unroll
                    for (int gx = 0; gx < G1 + 2; ++gx) {
                        if (gx < G1) {
                            const int qe = gstart[gbase + gx + 1];
                            int q = qs;
                            for (; q + 1 < qe; q += 2) {
                                PairRec r0, r1;
                                load_pair_rec(frec + q * CRS, r0);
                                load_pair_rec(frec + (q + 1) * CRS, r1);
                                accumulate_pair(r0, py, pz, M.h_inv, pa);
                                accumulate_pair(r1, py, pz, M.h_inv, pa);
                            }
                            if (q < qe) {
                                PairRec r0;
                                load_pair_rec(frec + q * CRS, r0);
                                accumulate_pair(r0, py, pz, M.h_inv, pa);
                            }
                            qs = qe;
                        }
                        const T a0[NC] = {pa[0].a01.x, pa[0].a01.y, pa[0].a23.x, pa[0].a23.y,
                                          pa[0].f01.x, pa[0].f01.y, pa[0].f2};
                        stage_node<NC, T>(part, pbase + gx, CSTR, a0);
                        pa[0] = pa[1];
                        pa[1] = pa[2];
                        pa[2].a01 = pa[2].a23 = pa[2].f01 = make_float2(0.f, 0.f);
                        pa[2].f2 = 0.f;
                    }
                } else {
                    T acc[3][NC];
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int c = 0; c < NC; ++c) acc[i][c] = T(0);
                    // The groups of the pencil in x order; two records of a group are
                    // loaded before either is accumulated. After group gx the x-node
                    // gx is final (later groups start further right).
                    int qs = gstart[gbase];
#pragma unroll
                    for (int gx = 0; gx < G1 + 2; ++gx) {
                        if (gx < G1) {
                            const int qe = gstart[gbase + gx + 1];
                            int q = qs;
                            if constexpr (MODE == 1) {
                                for (; q + 1 < qe; q += 2) {
                                    CompactRec<T> r0, r1;
                                    load_compact<D, T>(prec + q * CRS, r0);
                                    load_compact<D, T>(prec + (q + 1) * CRS, r1);
                                    accumulate_compact<D, T>(r0, py, pz, M.h_inv, acc);
                                    accumulate_compact<D, T>(r1, py, pz, M.h_inv, acc);
                                }
                                if (q < qe) {
                                    CompactRec<T> r0;
                                    load_compact<D, T>(prec + q * CRS, r0);
                                    accumulate_compact<D, T>(r0, py, pz, M.h_inv, acc);
                                }
                            } else {
                                for (; q + 1 < qe; q += 2) {
                                    PlainRec<T> r0, r1;
                                    load_plain<D, T>(prec + q * PRS, sj, sk, r0);
                                    load_plain<D, T>(prec + (q + 1) * PRS, sj, sk, r1);
                                    accumulate_plain<D, T>(r0, acc);
                                    accumulate_plain<D, T>(r1, acc);
                                }
                                if (q < qe) {
                                    PlainRec<T> r0;
                                    load_plain<D, T>(prec + q * PRS, sj, sk, r0);
                                    accumulate_plain<D, T>(r0, acc);
                                }
                            }
                            qs = qe;
                        }
                        stage_node<NC, T>(part, pbase + gx, CSTR, acc[0]);
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            acc[0][c] = acc[1][c];
                            acc[1][c] = acc[2][c];
                            acc[2][c] = T(0);
                        }
                    }
                }
            }
            __syncthreads();
            // ---- 3. per tile node: sum the staged partials (FP64), add to the grid
            for (int t = tid; t < TN; t += NT) {
                int node[3], tn[3] = {0, 0, 0}, rem = t;
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
                        const int pc = gy + G1 * gz;
                        const int idx = ((jj + 3 * kk) * NPENCIL + pc) * TS + tn[0];
#pragma unroll
                        for (int c = 0; c < NC; ++c) val[c] += double(part[idx + c * CSTR]);
                    }
#pragma unroll
                for (int d = 0; d < D; ++d) val[1 + D + d] += double(s.g[d]) * val[0];
                grid_add<D>(G, M, err, node[0], node[1], D == 3 ? node[2] : 0, val);
            }
        }
    };

    if constexpr (MODE == 2) {
        const int nlist = int(*bnd_count);
        for (int q = blockIdx.x; q < nlist; q += gridDim.x) process_block(bnd[q], 0, 1);
    } else {
        const int split = block_split(totals, NR);
        for (int vi = blockIdx.x; vi < nactive * split; vi += gridDim.x) {
            const int bi = split == 1 ? vi : vi / split, piece = vi - bi * split;
            const int b = blocklist[bi] - 1;
            if constexpr (MODE == 1) {
                if (!interior_block(b)) {  // the boundary launch's block (uniform over the CTA)
                    if (tid == 0 && piece == 0) bnd[atomicAdd(bnd_count, 1ull)] = b;
                    continue;
                }
            }
            process_block(b, piece, split);
        }
    }
}

// ---------------------------------------------------------------------------
// Plane kernel: the interior blocks of the 3D FP32 forms (quadratic B-spline,
// KernelCorrection(BSpline) whose interior windows are the plain kernel), with
// compact records in the packed FP32x2 layout (PairRec). The schedule of the
// pencil kernel with a wider lane: a lane owns one z-slot k of a pencil's
// window, i.e. the 3 x 3 (x, y) nodes of 3 window rows, and walks the pencil's
// groups in x order keeping the 3 x-slots x 3 rows x 7 components (63 FP32
// accumulators) in registers. Per record a lane loads the record once and
// evaluates the x and y jets once for 9 nodes instead of 3, so the per-record
// overhead (loads, jets, row factors) is paid 3 times per particle instead of
// 9; the 25 pencils x 3 z-slots are 75 lanes of the 128-thread CTA. After each
// group the x-node the window leaves for good is staged (3 rows, 7 components)
// to the lane's own slots of the staging array; one thread per tile node then
// sums the at most 9 staged partials in FP32 and adds the node to the grid
// with one global atomic per non-zero value. Every other block of the block
// list is appended to `bnd` for the full-record launch (MODE 2).
constexpr int PLANE_THREADS = 128;
constexpr int PLANE_NR = 512;

// One record's contribution to a plane lane's 3 x 3 nodes.
__device__ __forceinline__ void accumulate_plane(const PairRec& o, const SlotPoly& pz, float h_inv,
                                                 PairAcc (&acc)[3][3]) {
    const float tx = o.txy.x, ty = o.txy.y, tz = o.s5z.y;
    const float2 t2 = make_float2(tx, tx);
    // (wx_i, wx_i) and (dx_i, dx_i): the B-spline factors of the three x slots
    const float2 wx0 = __ffma2_rn(t2, __ffma2_rn(t2, make_float2(0.5f, 0.5f), make_float2(-1.f, -1.f)),
                                  make_float2(0.5f, 0.5f));
    const float2 wx1 = __ffma2_rn(t2, __ffma2_rn(t2, make_float2(-1.f, -1.f), make_float2(1.f, 1.f)),
                                  make_float2(0.5f, 0.5f));
    const float2 wx2 = __fmul2_rn(t2, __fmul2_rn(t2, make_float2(0.5f, 0.5f)));
    const float2 hh = make_float2(h_inv, h_inv);
    const float2 dx0 = __fmul2_rn(__fadd2_rn(t2, make_float2(-1.f, -1.f)), hh);
    const float2 dx1 = __fmul2_rn(__ffma2_rn(t2, make_float2(-2.f, -2.f), make_float2(1.f, 1.f)), hh);
    const float2 dx2 = __fmul2_rn(t2, hh);
    const float2 wxs[3] = {wx0, wx1, wx2}, dxs[3] = {dx0, dx1, dx2};
    // y jets of the three window rows, z jet of this lane's slot
    const float wy[3] = {0.5f + ty * (-1.0f + ty * 0.5f), 0.5f + ty * (1.0f + ty * -1.0f), ty * (ty * 0.5f)};
    const float dy[3] = {(-1.0f + ty) * h_inv, (1.0f + ty * -2.0f) * h_inv, ty * h_inv};
    const float wz = pz.a + tz * (pz.b + tz * pz.c);
    const float dz = (pz.e + tz * pz.f) * h_inv;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float wyz = wy[j] * wz, dyz = dy[j] * wz, wdz = wy[j] * dz;
        const float2 WYZ = make_float2(wyz, wyz);
        const float2 fa01 = __fmul2_rn(o.sa, WYZ);
        // the row's (m, m v) times wyz once; each x-slot then needs one FMA per pair
        const float2 m0j = __fmul2_rn(o.m0, WYZ), m1j = __fmul2_rn(o.m1, WYZ);
        const float2 fb01 = __ffma2_rn(o.sc, make_float2(wdz, wdz), __fmul2_rn(o.sb, make_float2(dyz, dyz)));
        const float fa2 = o.sc.x * wyz;
        const float fb2 = __fmaf_rn(o.s5z.x, wdz, o.sc.y * dyz);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            acc[i][j].a01 = __ffma2_rn(wxs[i], m0j, acc[i][j].a01);
            acc[i][j].a23 = __ffma2_rn(wxs[i], m1j, acc[i][j].a23);
            acc[i][j].f01 = __ffma2_rn(dxs[i], fa01, __ffma2_rn(wxs[i], fb01, acc[i][j].f01));
            acc[i][j].f2 = __fmaf_rn(dxs[i].x, fa2, __fmaf_rn(wxs[i].x, fb2, acc[i][j].f2));
        }
    }
}

template <bool X64>
__global__ void __launch_bounds__(PLANE_THREADS, 3)
    p2g_plane_kernel(DMesh<3, float> M, PView<float> P, GView<float> G, Scalars<float> s,
                     const int* __restrict__ totals, const int* __restrict__ blocklist,
                     const int* __restrict__ offsets, const int* __restrict__ perm, int* err,
                     int* __restrict__ bnd, unsigned long long* __restrict__ bnd_count) {
    using SH = PencilShape<3, 4>;
    constexpr int NT = PLANE_THREADS, NR = PLANE_NR, ITEMS = NR / NT;
    constexpr int TS = SH::TS, TN = SH::TN, NC = SH::NC, G1 = SH::G1, NG = SH::NG;
    constexpr int NJK = SH::NJK, NPENCIL = SH::NPENCIL;
    constexpr int CSTR = NPENCIL * NJK * TS;  // stride between components in the staging array
    constexpr int SKW = 2;                    // record skew per pencil (words)
    static_assert(NR % NT == 0 && NT % 8 == 0, "whole items per thread, passes in 8-particle chunks");
    static_assert(3 * NPENCIL <= NT, "one plane lane per (pencil, z slot)");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* rec = reinterpret_cast<float*>(smem_raw);
    // staged partials as (m, m v_x), (m v_y, m v_z), (f_x, f_y) pairs, then f_z:
    // [pair][jk][pencil][x] float2 and [jk][pencil][x] float (8-byte aligned)
    float* part = rec + NR * CRS + SKW * NPENCIL;
    float2* part2 = reinterpret_cast<float2*>(part);
    float* partz = part + 6 * CSTR;
    int* gcount = reinterpret_cast<int*>(part + NC * CSTR);
    int* gstart = gcount + NG;
    int* pslot = gstart + NG + 1;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nactive = totals[0];

    for (int g = tid; g < NG; g += NT) gcount[g] = 0;
    __syncthreads();

    const int split = block_split(totals, NR);
    for (int vi = blockIdx.x; vi < nactive * split; vi += gridDim.x) {
        const int bi = split == 1 ? vi : vi / split, piece = vi - bi * split;
        const int b = blocklist[bi] - 1;
        int org[3];
        bool interior = true;
        {
            int r = b;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                org[d] = (r % M.nb[d]) * 4 - 1;
                r /= M.nb[d];
                interior = interior && org[d] >= 0 && org[d] + TS - 1 <= M.n[d] - 1;
            }
        }
        if (!interior) {  // the full-record launch's block (uniform over the CTA)
            if (tid == 0 && piece == 0) bnd[atomicAdd(bnd_count, 1ull)] = b;
            continue;
        }
        const int s0 = offsets[b], s1 = offsets[b + 1];
        const BlockPasses bp(s0, s1, NR);
        for (int bi = piece; bi < bp.count(); bi += split) {
            const int q0 = bp.pos(bi, tid), qstep = bp.step(NT);
            // ---- 1a. every global load of the batch first, then group and rank;
            //      the record's 14 values stay in registers until the slot is known
            int pid[ITEMS], grp[ITEMS], rank[ITEMS];
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                const int ti = tid + u * NT, q = q0 + u * qstep;
                pid[u] = (ti < NR && q < s1) ? perm[q] - 1 : -1;
            }
            float pv[ITEMS][3], pV[ITEMS], pm[ITEMS], psg[ITEMS][6], pt[ITEMS][3];
            double pxd[ITEMS][3];
            float pxf[ITEMS][3];
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                const long long p = pid[u] >= 0 ? pid[u] : 0;
                const bool on = pid[u] >= 0;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if constexpr (X64) pxd[u][d] = on ? P.x64[d][p] : 0.0;
                    else pxf[u][d] = on ? P.x[d][p] : 0.0f;
                    pv[u][d] = on ? P.v[d][p] : 0.0f;
                }
                pV[u] = on ? P.V[p] : 0.0f;
                pm[u] = (on && P.m) ? P.m[p] : s.mass;
#pragma unroll
                for (int k = 0; k < 6; ++k) psg[u][k] = on ? P.sig[k][p] : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                grp[u] = -1;
                rank[u] = 0;
                if (pid[u] < 0) continue;
                int gi = 0;
                bool ok = true;
#pragma unroll
                for (int d = 2; d >= 0; --d) {
                    // window start floor(xi - 1/2) and the fast path's t = fract(xi - 1/2)
                    // (bspline.jl:28-40, 90-100)
                    int lo;
                    if constexpr (X64) {
                        const double u64 = (pxd[u][d] - M.xmin64[d]) * M.h_inv64 - 0.5;
                        const double fl = floor(u64);
                        lo = int(fl);
                        float t = float(u64 - fl);
                        if (t >= 1.0f) t = 1.0f - 1.0f / float(1 << 24);
                        pt[u][d] = t;
                    } else {
                        const float uu = (pxf[u][d] - M.xmin[d]) * M.h_inv - 0.5f;
                        const float fl = floorf(uu);
                        lo = int(fl);
                        pt[u][d] = uu - fl;
                    }
                    const int q = lo - org[d];
                    ok = ok && q >= 0 && q < G1;
                    gi = gi * G1 + q;
                }
                if (!ok) {
                    atomicOr(err, ERR_TILE_RANGE);
                    continue;
                }
                grp[u] = gi;
                rank[u] = atomicAdd(&gcount[gi], 1);
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
            } else if (warp == 1) {
                // pencil slots by size, largest first: the pencils of one warp
                // then have similar lengths
                const int myp = lane < NPENCIL ? lane : -1;
                int mysize = 0;
                if (myp >= 0) {
                    const int gb = G1 * myp;
#pragma unroll
                    for (int gx = 0; gx < G1; ++gx) mysize += gcount[gb + gx];
                }
                int rk = 0;
                for (int o = 0; o < NPENCIL; ++o) {
                    const int os = __shfl_sync(0xffffffffu, mysize, o);
                    rk += (os > mysize) || (os == mysize && o < lane);
                }
                if (myp >= 0) pslot[rk] = myp;
            }
            __syncthreads();
            // ---- 1b. records at their group-sorted slots (PairRec layout)
            for (int g = tid; g < NG; g += NT) gcount[g] = 0;  // ready for the next batch
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                if (grp[u] < 0) continue;
                float* r = rec + (gstart[grp[u]] + rank[u]) * CRS + SKW * (grp[u] / G1);
                const float mp = pm[u], nV = -pV[u];
                st2(r + 0, mp, mp * pv[u][0]);
                st2(r + 2, mp * pv[u][1], mp * pv[u][2]);
                st2(r + 4, nV * psg[u][0], nV * psg[u][1]);
                st2(r + 6, nV * psg[u][1], nV * psg[u][3]);
                st2(r + 8, nV * psg[u][2], nV * psg[u][4]);
                st2(r + 10, nV * psg[u][5], pt[u][2]);
                st2(r + 12, pt[u][0], pt[u][1]);
            }
            __syncthreads();
            // ---- 2. plane sweeps: lane (pencil slot, z slot k)
            if (tid < 3 * NPENCIL) {
                const int slot = tid / 3, k = tid - 3 * slot;
                const int pc = pslot[slot];
                const int gbase = G1 * pc;
                const float* prec = rec + SKW * pc;
                const SlotPoly pz = slot_poly(k);
                PairAcc acc[3][3];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        acc[i][j].a01 = acc[i][j].a23 = acc[i][j].f01 = make_float2(0.f, 0.f);
                        acc[i][j].f2 = 0.f;
                    }
                int qs = gstart[gbase];
#pragma unroll
                for (int gx = 0; gx < G1 + 2; ++gx) {
                    if (gx < G1) {
                        const int qe = gstart[gbase + gx + 1];
#pragma unroll 1
                        for (int q = qs; q < qe; ++q) {
                            PairRec r0;
                            load_pair_rec(prec + q * CRS, r0);
                            accumulate_plane(r0, pz, M.h_inv, acc);
                        }
                        qs = qe;
                    }
                    // x-node gx of rows (j, k) is final: stage it, shift the rows
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const int o = ((j + 3 * k) * NPENCIL + pc) * TS + gx;
                        part2[o] = acc[0][j].a01;
                        part2[CSTR + o] = acc[0][j].a23;
                        part2[2 * CSTR + o] = acc[0][j].f01;
                        partz[o] = acc[0][j].f2;
                        acc[0][j] = acc[1][j];
                        acc[1][j] = acc[2][j];
                        acc[2][j].a01 = acc[2][j].a23 = acc[2][j].f01 = make_float2(0.f, 0.f);
                        acc[2][j].f2 = 0.f;
                    }
                }
            }
            __syncthreads();
            // ---- 3. per tile node: FP32 sum of the staged partials, one global
            //      atomic per non-zero value (gravity from the summed mass)
            for (int t = tid; t < TN; t += NT) {
                const int tx = t % TS, ty = (t / TS) % TS, tz = t / (TS * TS);
                float2 a01 = make_float2(0.f, 0.f), a23 = a01, f01 = a01;
                float f2 = 0.f;
#pragma unroll
                for (int kk = 0; kk < 3; ++kk)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj) {
                        const int gy = ty - jj, gz = tz - kk;
                        if (gy < 0 || gy >= G1 || gz < 0 || gz >= G1) continue;
                        const int idx = ((jj + 3 * kk) * NPENCIL + gy + G1 * gz) * TS + tx;
                        const float2 p0 = part2[idx], p1 = part2[CSTR + idx], p2 = part2[2 * CSTR + idx];
                        a01.x += p0.x;
                        a01.y += p0.y;
                        a23.x += p1.x;
                        a23.y += p1.y;
                        f01.x += p2.x;
                        f01.y += p2.y;
                        f2 += partz[idx];
                    }
                float val[NC] = {a01.x, a01.y, a23.x, a23.y, f01.x, f01.y, f2};
#pragma unroll
                for (int d = 0; d < 3; ++d) val[4 + d] += s.g[d] * val[0];
                grid_add<3>(G, M, err, org[0] + tx, org[1] + ty, org[2] + tz, val);
            }
        }
    }
}

size_t plane_smem_bytes() {
    using SH = PencilShape<3, 4>;
    return sizeof(float) * (size_t(PLANE_NR) * CRS + 2 * SH::NPENCIL + SH::NPART) +
           sizeof(int) * size_t(SH::NG + SH::NG + 1 + 32);
}

template <bool X64>
cudaError_t launch_plane(const DMesh<3, float>& M, const PView<float>& P, const GView<float>& G,
                         const Scalars<float>& s, const BinBuffers& b, const LaunchCfg& cfg) {
    auto kern = p2g_plane_kernel<X64>;
    const size_t smem = plane_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, int(cudaSharedmemCarveoutMaxShared));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PLANE_THREADS, smem);
    const int grid = std::min(cfg.num_sms * std::max(per_sm, 1), 8 * M.nblocks);  // blocks may be split (block_split)
    kern<<<grid, PLANE_THREADS, smem, cfg.stream>>>(M, P, G, s, b.totals, b.blocklist, b.offsets, b.perm, cfg.err,
                                                   b.cursors, b.partials);
    ++*cfg.launches;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// General plane kernel (3D): WLS weights (wls.jl:51-84) and/or the APIC affine
// term mv_i += w_i m_p (v_p + B_p D^-1 (x_i - x_p)) (docs/src/transfer.md:
// 176-178, D^-1 = 4/h^2 I), on the plane-lane schedule of p2g_plane_kernel.
// Every quantity is a product of axis factors with an affine function of the
// node offset r = X_i - x_p, so a lane evaluates it per window row from a few
// per-row constants:
//   WLS:  N_i = w_i (Mi[0] . P_i), grad N_i = w_i (Mi[1..3] . P_i), P = (1, r),
//         w_i = wx wy wz the kernel (uGIMP or B-spline) values;
//         per row j: A = Mi00 + Mi02 ry + Mi03 rz, C_d = Mi_d0 + Mi_d2 ry + Mi_d3 rz,
//         per node:  N = w (A + Mi01 rx), G_d = w (C_d + Mi_d1 rx);
//   plain kernel: N = w, G = the kernel jets' gradient;
//   APIC: per row U = (m D^-1 B)[:,1] ry + (m D^-1 B)[:,2] rz, per node
//         mv += N (m v_p + U + (m D^-1 B)[:,0] rx).
// Records hold m_p, m_p v_p, -V_p sigma_p, the axis kernel values (and their
// derivatives without WLS), r0 = X_lo - x_p per axis, the symmetric moment
// inverse (WLS) and m_p D^-1 B_p (APIC). Any block (windows truncated at the
// mesh boundary have zero values on their missing slots); staging and the
// per-node gather as in p2g_plane_kernel, in T.
template <bool WLSF, bool APICF>
struct GenRec {
    static constexpr int M = 0, MV = 1, S = 4, W = 10;  // W: kernel values x[3] y[3] z[3]
    static constexpr int DW = 19;                       // without WLS: derivative jets x[3] y[3] z[3] (times h_inv)
    static constexpr int R0 = WLSF ? 19 : 28;           // X_lo - x_p per axis
    static constexpr int MI = R0 + 3;                   // WLS: Mi 00 01 02 03 11 12 13 22 23 33
    static constexpr int DB = MI + (WLSF ? 10 : 0);     // APIC: m D^-1 B, column-major
    static constexpr int END = DB + (APICF ? 9 : 0);
    static constexpr int SIZE = (END + 1) & ~1;
};

constexpr int GEN_THREADS = 128;

template <class T, bool X64, bool WLSF, bool APICF, int NR>
__global__ void __launch_bounds__(GEN_THREADS, sizeof(T) == 4 ? 2 : 1)
    p2g_gen_plane_kernel(DMesh<3, T> M, PView<T> P, GView<T> G, Scalars<T> s, const int* __restrict__ totals,
                         const int* __restrict__ blocklist, const int* __restrict__ offsets,
                         const int* __restrict__ perm, int* err) {
    using SH = PencilShape<3, 4>;
    using R = GenRec<WLSF, APICF>;
    constexpr int NT = GEN_THREADS, ITEMS = NR / NT, RS = R::SIZE;
    constexpr int TS = SH::TS, TN = SH::TN, NC = SH::NC, G1 = SH::G1, NG = SH::NG;
    constexpr int NJK = SH::NJK, NPENCIL = SH::NPENCIL;
    constexpr int CSTR = NPENCIL * NJK * TS;
    constexpr int SKW = 2;
    static_assert(NR % NT == 0 && NT % 8 == 0, "whole items per thread, passes in 8-particle chunks");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* rec = reinterpret_cast<T*>(smem_raw);
    T* part = rec + NR * RS + SKW * NPENCIL;
    int* gcount = reinterpret_cast<int*>(part + NC * CSTR);
    int* gstart = gcount + NG;
    int* pslot = gstart + NG + 1;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nactive = totals[0];
    const T h = M.h;
    const T dinv = T(4) / (M.h * M.h);

    for (int g = tid; g < NG; g += NT) gcount[g] = 0;
    __syncthreads();

    const int split = block_split(totals, NR);
    for (int vi = blockIdx.x; vi < nactive * split; vi += gridDim.x) {
        const int bi = split == 1 ? vi : vi / split, piece = vi - bi * split;
        const int b = blocklist[bi] - 1;
        int org[3];
        {
            int r = b;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                org[d] = (r % M.nb[d]) * 4 - 1;
                r /= M.nb[d];
            }
        }
        const int s0 = offsets[b], s1 = offsets[b + 1];
        const BlockPasses bp(s0, s1, NR);
        for (int bi = piece; bi < bp.count(); bi += split) {
            const int q0 = bp.pos(bi, tid), qstep = bp.step(NT);
            // ---- 1a. window start -> group and rank
            int pid[ITEMS], grp[ITEMS], rank[ITEMS];
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                const int ti = tid + u * NT, q = q0 + u * qstep;
                pid[u] = (ti < NR && q < s1) ? perm[q] - 1 : -1;
                grp[u] = -1;
                rank[u] = 0;
            }
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                if (pid[u] < 0) continue;
                const long long p = pid[u];
                const T l = P.l ? P.l[p] : s.gimp_l;
                int lo[3], cnt[3];
                bool inside;
                if constexpr (X64) {
                    double x[3], xi[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) x[d] = P.x64[d][p];
                    inside = axis_window_x64<3, T>(M, s.basis, x, double(l) / M.h64, xi, lo, cnt);
                } else {
                    T x[3], xi[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) x[d] = P.x[d][p];
                    inside = axis_window<3, T>(M, s.basis, x, l / M.h, xi, lo, cnt);
                }
                if (!inside) continue;
                int gi = 0;
                bool ok = true;
#pragma unroll
                for (int d = 2; d >= 0; --d) {
                    const int q = lo[d] - org[d];
                    ok = ok && q >= 0 && q < G1;
                    gi = gi * G1 + q;
                }
                if (!ok) {
                    atomicOr(err, ERR_TILE_RANGE);
                    continue;
                }
                grp[u] = gi;
                rank[u] = atomicAdd(&gcount[gi], 1);
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
            } else if (warp == 1) {
                const int myp = lane < NPENCIL ? lane : -1;
                int mysize = 0;
                if (myp >= 0) {
                    const int gb = G1 * myp;
#pragma unroll
                    for (int gx = 0; gx < G1; ++gx) mysize += gcount[gb + gx];
                }
                int rk = 0;
                for (int o = 0; o < NPENCIL; ++o) {
                    const int os = __shfl_sync(0xffffffffu, mysize, o);
                    rk += (os > mysize) || (os == mysize && o < lane);
                }
                if (myp >= 0) pslot[rk] = myp;
            }
            __syncthreads();
            // ---- 1b. basis (kernel jets, WLS moment inverse) and the record
            for (int g = tid; g < NG; g += NT) gcount[g] = 0;
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                if (grp[u] < 0) continue;
                const long long p = pid[u];
                const T l = P.l ? P.l[p] : s.gimp_l;
                Basis<3, T> B;
                T r0[3];
                if constexpr (X64) {
                    double x[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) x[d] = P.x64[d][p];
                    prepare_basis_x64<3, T, WLSF>(M, s.basis, x, l, B, err);
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        r0[d] = T(__dadd_rn(M.xmin64[d], __dmul_rn(double(B.ax[d].lo), M.h64)) - x[d]);
                } else {
                    T x[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) x[d] = P.x[d][p];
                    prepare_basis<3, T, WLSF>(M, s.basis, x, l, B, err);
#pragma unroll
                    for (int d = 0; d < 3; ++d) r0[d] = node_coord(M, d, B.ax[d].lo) - x[d];
                }
                T* rr = rec + (gstart[grp[u]] + rank[u]) * RS + SKW * (grp[u] / G1);
                const T mp = P.m ? P.m[p] : s.mass;
                const T nV = -P.V[p];
                rr[R::M] = mp;
#pragma unroll
                for (int d = 0; d < 3; ++d) rr[R::MV + d] = mp * P.v[d][p];
#pragma unroll
                for (int k = 0; k < 6; ++k) rr[R::S + k] = nV * P.sig[k][p];
#pragma unroll
                for (int d = 0; d < 3; ++d)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        rr[R::W + 3 * d + k] = B.ax[d].val[k];
                        if constexpr (!WLSF) rr[R::DW + 3 * d + k] = B.ax[d].der[k] * M.h_inv;
                    }
#pragma unroll
                for (int d = 0; d < 3; ++d) rr[R::R0 + d] = r0[d];
                if constexpr (WLSF) {
                    rr[R::MI + 0] = B.Mi[0][0];
                    rr[R::MI + 1] = B.Mi[0][1];
                    rr[R::MI + 2] = B.Mi[0][2];
                    rr[R::MI + 3] = B.Mi[0][3];
                    rr[R::MI + 4] = B.Mi[1][1];
                    rr[R::MI + 5] = B.Mi[1][2];
                    rr[R::MI + 6] = B.Mi[1][3];
                    rr[R::MI + 7] = B.Mi[2][2];
                    rr[R::MI + 8] = B.Mi[2][3];
                    rr[R::MI + 9] = B.Mi[3][3];
                }
                if constexpr (APICF) {
                    const T md = mp * dinv;
#pragma unroll
                    for (int k = 0; k < 9; ++k) rr[R::DB + k] = md * P.B[k][p];
                }
            }
            __syncthreads();
            // ---- 2. plane sweeps: lane (pencil slot, z slot k)
            if (tid < 3 * NPENCIL) {
                const int slot = tid / 3, k = tid - 3 * slot;
                const int pc = pslot[slot];
                const int gbase = G1 * pc;
                const T* prec = rec + SKW * pc;
                T acc[3][3][NC];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
#pragma unroll
                        for (int c = 0; c < NC; ++c) acc[i][j][c] = T(0);
                int qs = gstart[gbase];
#pragma unroll
                for (int gx = 0; gx < G1 + 2; ++gx) {
                    if (gx < G1) {
                        const int qe = gstart[gbase + gx + 1];
                        for (int q = qs; q < qe; ++q) {
                            const T* r = prec + q * RS;
                            const T mp = r[R::M];
                            const T mv[3] = {r[R::MV], r[R::MV + 1], r[R::MV + 2]};
                            const T S[6] = {r[R::S], r[R::S + 1], r[R::S + 2], r[R::S + 3], r[R::S + 4], r[R::S + 5]};
                            const T wz = r[R::W + 6 + k];
                            const T rz = r[R::R0 + 2] + T(k) * h;
                            T mi[10] = {}, db[9] = {}, dz = T(0);
                            if constexpr (WLSF) {
#pragma unroll
                                for (int c = 0; c < 10; ++c) mi[c] = r[R::MI + c];
                            } else {
                                dz = r[R::DW + 6 + k];
                            }
                            if constexpr (APICF) {
#pragma unroll
                                for (int c = 0; c < 9; ++c) db[c] = r[R::DB + c];
                            }
#pragma unroll
                            for (int j = 0; j < 3; ++j) {
                                const T ry = r[R::R0 + 1] + T(j) * h;
                                const T wyz = r[R::W + 3 + j] * wz;
                                // per-row constants
                                T A = T(0), Cd[3] = {T(0), T(0), T(0)}, dyz = T(0), wdz = T(0);
                                if constexpr (WLSF) {
                                    A = mi[0] + mi[2] * ry + mi[3] * rz;
                                    Cd[0] = mi[1] + mi[5] * ry + mi[6] * rz;  // row 1: Mi10 Mi11 Mi12 Mi13
                                    Cd[1] = mi[2] + mi[7] * ry + mi[8] * rz;  // row 2: Mi20 Mi21 Mi22 Mi23
                                    Cd[2] = mi[3] + mi[8] * ry + mi[9] * rz;  // row 3: Mi30 Mi31 Mi32 Mi33
                                } else {
                                    dyz = r[R::DW + 3 + j] * wz;
                                    wdz = r[R::W + 3 + j] * dz;
                                }
                                T U[3] = {mv[0], mv[1], mv[2]};
                                if constexpr (APICF) {
#pragma unroll
                                    for (int a = 0; a < 3; ++a) U[a] += db[a + 3] * ry + db[a + 6] * rz;
                                }
#pragma unroll
                                for (int i = 0; i < 3; ++i) {
                                    const T rx = r[R::R0] + T(i) * h;
                                    const T wx = r[R::W + i];
                                    const T w = wx * wyz;
                                    T N, Gd[3];
                                    if constexpr (WLSF) {
                                        N = w * (A + mi[1] * rx);
                                        Gd[0] = w * (Cd[0] + mi[4] * rx);
                                        Gd[1] = w * (Cd[1] + mi[5] * rx);
                                        Gd[2] = w * (Cd[2] + mi[6] * rx);
                                    } else {
                                        N = w;
                                        Gd[0] = r[R::DW + i] * wyz;
                                        Gd[1] = wx * dyz;
                                        Gd[2] = wx * wdz;
                                    }
                                    acc[i][j][0] += N * mp;
#pragma unroll
                                    for (int a = 0; a < 3; ++a) {
                                        T va = U[a];
                                        if constexpr (APICF) va += db[a] * rx;
                                        acc[i][j][1 + a] += N * va;
                                    }
                                    acc[i][j][4] += S[0] * Gd[0] + S[1] * Gd[1] + S[2] * Gd[2];
                                    acc[i][j][5] += S[1] * Gd[0] + S[3] * Gd[1] + S[4] * Gd[2];
                                    acc[i][j][6] += S[2] * Gd[0] + S[4] * Gd[1] + S[5] * Gd[2];
                                }
                            }
                        }
                        qs = qe;
                    }
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        T* dst = part + ((j + 3 * k) * NPENCIL + pc) * TS + gx;
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            dst[c * CSTR] = acc[0][j][c];
                            acc[0][j][c] = acc[1][j][c];
                            acc[1][j][c] = acc[2][j][c];
                            acc[2][j][c] = T(0);
                        }
                    }
                }
            }
            __syncthreads();
            // ---- 3. per tile node inside the mesh: sum of the staged partials
            for (int t = tid; t < TN; t += NT) {
                const int tx = t % TS, ty = (t / TS) % TS, tz = t / (TS * TS);
                const int nx = org[0] + tx, ny = org[1] + ty, nz = org[2] + tz;
                if (nx < 0 || ny < 0 || nz < 0 || nx >= M.n[0] || ny >= M.n[1] || nz >= M.n[2]) continue;
                T val[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) val[c] = T(0);
#pragma unroll
                for (int kk = 0; kk < 3; ++kk)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj) {
                        const int gy = ty - jj, gz = tz - kk;
                        if (gy < 0 || gy >= G1 || gz < 0 || gz >= G1) continue;
                        const int idx = ((jj + 3 * kk) * NPENCIL + gy + G1 * gz) * TS + tx;
#pragma unroll
                        for (int c = 0; c < NC; ++c) val[c] += part[idx + c * CSTR];
                    }
#pragma unroll
                for (int d = 0; d < 3; ++d) val[4 + d] += s.g[d] * val[0];
                grid_add<3>(G, M, err, nx, ny, nz, val);
            }
        }
    }
}

template <class T, bool WLSF, bool APICF, int NR>
size_t gen_smem_bytes() {
    using SH = PencilShape<3, 4>;
    return sizeof(T) * (size_t(NR) * GenRec<WLSF, APICF>::SIZE + 2 * SH::NPENCIL + SH::NPART) +
           sizeof(int) * size_t(SH::NG + SH::NG + 1 + 32);
}

template <class T, bool X64, bool WLSF, bool APICF>
cudaError_t launch_gen_plane_t(const DMesh<3, T>& M, const PView<T>& P, const GView<T>& G, const Scalars<T>& s,
                               const BinBuffers& b, const LaunchCfg& cfg) {
    // Records per batch: 256 in FP32 (2 CTAs per SM), 128 in FP64.
    constexpr int NR = sizeof(T) == 4 ? 256 : 128;
    auto kern = p2g_gen_plane_kernel<T, X64, WLSF, APICF, NR>;
    const size_t smem = gen_smem_bytes<T, WLSF, APICF, NR>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, int(cudaSharedmemCarveoutMaxShared));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, GEN_THREADS, smem);
    const int grid = std::min(cfg.num_sms * std::max(per_sm, 1), 8 * M.nblocks);  // blocks may be split (block_split)
    KernelScope ks(cfg, "p2g");
    kern<<<grid, GEN_THREADS, smem, cfg.stream>>>(M, P, G, s, b.totals, b.blocklist, b.offsets, b.perm, cfg.err);
    ++*cfg.launches;
    return cudaGetLastError();
}

template <class T, bool X64>
cudaError_t launch_gen_plane(const DMesh<3, T>& M, const PView<T>& P, const GView<T>& G, const Scalars<T>& s,
                             const BinBuffers& b, const LaunchCfg& cfg) {
    const bool wls = s.basis == TB_WLS_BSPLINE_QUADRATIC || s.basis == TB_WLS_UGIMP;
    const bool apic = s.transfer == TB_TRANSFER_APIC;
    if (wls && apic) return launch_gen_plane_t<T, X64, true, true>(M, P, G, s, b, cfg);
    if (wls) return launch_gen_plane_t<T, X64, true, false>(M, P, G, s, b, cfg);
    return launch_gen_plane_t<T, X64, false, true>(M, P, G, s, b, cfg);
}

template <int D, class T, int BW, int NR, int MODE>
size_t pencil_smem_bytes() {
    using SH = PencilShape<D, BW>;
    const int rs = (MODE == 1) ? CRS : PRS;
    return sizeof(T) * (size_t(NR) * rs + SH::skew(MODE, sizeof(T)) * SH::NPENCIL + SH::NPART) +
           sizeof(int) * size_t(SH::NG + SH::NG + 1 + 32);
}

template <int D, class T, int BW, bool X64, int MODE>
cudaError_t launch_pencil_mode(const DMesh<D, T>& M, const PView<T>& P, const GView<T>& G, const Scalars<T>& s,
                               const BinBuffers& b, const LaunchCfg& cfg) {
    // Records per batch: a whole cube3d block (512). FP32 full records: 2 CTAs per
    // SM (103 KB of shared memory); compact records: 3 (72 KB); FP64: 1.
    constexpr int NR = 512;
    auto kern = p2g_pencil_kernel<D, T, BW, NR, X64, MODE>;
    const size_t smem = pencil_smem_bytes<D, T, BW, NR, MODE>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, int(cudaSharedmemCarveoutMaxShared));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, P2G_THREADS, smem);
    const int grid = std::min(cfg.num_sms * std::max(per_sm, 1), 8 * M.nblocks);  // blocks may be split (block_split)
    // the boundary-block list lives in binning scratch that is free until the
    // next binning: cursors (one int per block) and the first scan partial
    kern<<<grid, P2G_THREADS, smem, cfg.stream>>>(M, P, G, s, b.totals, b.blocklist, b.offsets, b.perm, cfg.err,
                                                 b.cursors, b.partials);
    ++*cfg.launches;
    return cudaGetLastError();
}

// The quadratic B-spline in the FP32 forms runs two launches: compact records on
// the interior blocks, full records on the blocks at the mesh boundary (their
// windows may be truncated). Other bases and FP64 run one full-record launch.
template <int D, class T, int BW, bool X64>
cudaError_t launch_pencil(const DMesh<D, T>& M, const PView<T>& P, const GView<T>& G, const Scalars<T>& s,
                          const BinBuffers& b, const LaunchCfg& cfg) {
    KernelScope ks(cfg, "p2g");
    if constexpr (sizeof(T) == 4) {
        if (s.basis == TB_BSPLINE_QUADRATIC || s.basis == TB_KC_BSPLINE_QUADRATIC) {
            cudaError_t e = cudaMemsetAsync(b.partials, 0, sizeof(unsigned long long), cfg.stream);
            if (e != cudaSuccess) return e;
            if constexpr (D == 3 && BW == 4) e = launch_plane<X64>(M, P, G, s, b, cfg);
            else e = launch_pencil_mode<D, T, BW, X64, 1>(M, P, G, s, b, cfg);
            if (e != cudaSuccess) return e;
            return launch_pencil_mode<D, T, BW, X64, 2>(M, P, G, s, b, cfg);
        }
    }
    return launch_pencil_mode<D, T, BW, X64, 0>(M, P, G, s, b, cfg);
}

template <int D, class T, int BW, bool GEN, int NR>
size_t p2g_smem_bytes() {
    constexpr int TS = BW + 3;
    constexpr int TN = (D == 3) ? TS * TS * TS : TS * TS;
    constexpr int NC = 1 + 2 * D;
    constexpr int NG = (D == 3) ? (BW + 1) * (BW + 1) * (BW + 1) : (BW + 1) * (BW + 1);
    const size_t tiles = tile_bytes<NC * TN>();
    const size_t recs = sizeof(T) * size_t(NR) * Rec<D, GEN>::SIZE;
    const size_t ints = sizeof(int) * size_t(NG + NG + 1 + 32);
    return tiles + recs + ints;
}

template <int D, class T, int BW, bool GEN>
cudaError_t launch_group(const DMesh<D, T>& M, const PView<T>& P, const GView<T>& G, const Scalars<T>& s,
                         const BinBuffers& b, const LaunchCfg& cfg) {
    // Records per batch: a whole cube3d block (512) in FP32, half of it in FP64
    // or with the general (WLS/APIC) record.
    constexpr int NR = (sizeof(T) == 4 && !GEN) ? 512 : 256;
    auto kern = p2g_group_kernel<D, T, BW, GEN, NR>;
    const size_t smem = p2g_smem_bytes<D, T, BW, GEN, NR>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, P2G_THREADS, smem);
    const int grid = std::min(cfg.num_sms * std::max(per_sm, 1), M.nblocks);
    KernelScope ks(cfg, "p2g");
    kern<<<grid, P2G_THREADS, smem, cfg.stream>>>(M, P, G, s, b.totals, b.blocklist, b.offsets, b.perm, cfg.err);
    ++*cfg.launches;
    return cudaGetLastError();
}

}  // namespace

template <int D, class T, int BW>
cudaError_t launch_p2g(const DMesh<D, T>& M, const PView<T>& P, const GView<T>& G, const Scalars<T>& s,
                       const BinBuffers& b, const LaunchCfg& cfg) {
    if (P.n == 0) return cudaSuccess;
    const bool gen = s.transfer == TB_TRANSFER_APIC || s.basis == TB_WLS_BSPLINE_QUADRATIC || s.basis == TB_WLS_UGIMP;
    if (P.x64[0]) {  // FP64-position form: FP32 state only (checked by the caller)
        if constexpr (sizeof(T) == 4) {
            if (!gen) return launch_pencil<D, T, BW, true>(M, P, G, s, b, cfg);
            if constexpr (D == 3 && BW == 4) return launch_gen_plane<T, true>(M, P, G, s, b, cfg);
        }
        return cudaErrorInvalidValue;
    }
    if (gen) {
        if constexpr (D == 3 && BW == 4) return launch_gen_plane<T, false>(M, P, G, s, b, cfg);
        return launch_group<D, T, BW, true>(M, P, G, s, b, cfg);
    }
    return launch_pencil<D, T, BW, false>(M, P, G, s, b, cfg);
}

#define TB_INST_P2G(D, T, BW)                                                                        \
    template cudaError_t launch_p2g<D, T, BW>(const DMesh<D, T>&, const PView<T>&, const GView<T>&, \
                                              const Scalars<T>&, const BinBuffers&, const LaunchCfg&);
TB_INST_P2G(3, double, 4)
TB_INST_P2G(3, float, 4)
TB_INST_P2G(2, double, 8)
TB_INST_P2G(2, float, 8)
TB_INST_P2G(2, double, 4)
TB_INST_P2G(2, float, 4)

}  // namespace tb
