// tb_p2g.cu -- block-scheduled P2G scatter of m, mv and f
// (Tesserae.jl src/Transfer/gpu.jl:139-223; equations README.md:72-74,
// test/transfer.jl:96-97 for gravity, docs/src/transfer.md:176-178 for APIC).
//
// One CTA per non-empty grid block (grid-stride over the device block list).
// The block's particles reach the (BW+3)^D-node halo tile [BW b - 1, BW b + BW + 1]
// per axis; every support window starts at one of (BW+1)^D tile positions.
//
// Per batch of up to NB particles of the block:
//   1. one thread per particle evaluates the basis once (per-axis values and
//      derivatives, zero past a truncated window) and writes a compact record
//      (sources m_p, v_p, -V_p sigma_p; axis jets; for WLS/APIC also x_p, the
//      moment inverse and B_p) to shared memory, and counting-sorts the batch by
//      window start ("group");
//   2. one warp per group maps lanes to the 3^D window nodes (2D: 9 nodes x 3
//      particle lanes) and streams the group's particles, reading each record by
//      broadcast and accumulating the node's m, mv, f in registers;
//   3. each lane adds its node sums into the shared tile once per group. Lanes
//      of a warp touch distinct nodes, so the only collisions are between warps.
//      FP32 adds are compensated: atomicAdd returns the old value, the rounding
//      error of old + x is recovered exactly (two-sum) into a second tile.
// After the last batch the tile is flushed with one global atomic per non-zero
// node value (gravity, sum w m g = g sum w m, is added there from the tile mass).
#include "tb_launch.cuh"

namespace tb {

namespace {

__device__ __forceinline__ void tile_add(double* hi, double*, int idx, double x) {
    if (x != 0.0) atomicAdd(&hi[idx], x);
}

__device__ __forceinline__ void tile_add(float* hi, float* lo, int idx, float x) {
    if (x == 0.0f) return;
    const float old = atomicAdd(&hi[idx], x);
    const float s = __fadd_rn(old, x);
    const float bp = __fsub_rn(s, old);
    const float e = __fadd_rn(__fsub_rn(old, __fsub_rn(s, bp)), __fsub_rn(x, bp));
    if (e != 0.0f) atomicAdd(&lo[idx], e);
}

// Record layout (in T words), padded to a multiple of 4:
//   [0]      m_p            [1..D]   v_p
//   [4..]    S = -V sigma (symmetric, nsym)   -> 4 .. 4+nsym
//   [AX..]   per axis d, per slot k: (value, derivative) -> AX + 6 d + 2 k
//   GEN only: [XP..] x_p (D), [MI..] moment inverse (D+1)^2, [BP..] B_p (D^2)
template <int D, bool GEN>
struct Rec {
    static constexpr int NS = (D == 3) ? 6 : 3;
    static constexpr int AX = 4 + ((NS + 3) / 4) * 4;  // 12 (3D), 8 (2D)
    static constexpr int XP = AX + 6 * D;
    static constexpr int MI = XP + 4;
    static constexpr int BP = MI + (D + 1) * (D + 1);
    static constexpr int END = GEN ? BP + D * D : XP;
    static constexpr int SIZE = ((END + 3) / 4) * 4;
};

template <int D, class T, int BW, bool GEN, int NB>
__global__ void __launch_bounds__(NB, 2) p2g_group_kernel(DMesh<D, T> M, PView<T> P, GView<T> G, Scalars<T> s,
                                                       const int* __restrict__ totals,
                                                       const int* __restrict__ blocklist,
                                                       const int* __restrict__ offsets,
                                                       const int* __restrict__ perm, int* err) {
    constexpr int TS = BW + 3;
    constexpr int TN = (D == 3) ? TS * TS * TS : TS * TS;
    constexpr int NC = 1 + 2 * D;
    constexpr bool COMP = sizeof(T) == 4;
    constexpr int G1 = BW + 1;  // window starts per axis
    constexpr int NG = (D == 3) ? G1 * G1 * G1 : G1 * G1;
    constexpr int NSLOT = (D == 3) ? 27 : 9;
    constexpr int NSUB = 32 / NSLOT;  // particle lanes per slot (1 in 3D, 3 in 2D)
    constexpr int RS = Rec<D, GEN>::SIZE;
    constexpr int NW = NB / 32;
    using R = Rec<D, GEN>;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* hi = reinterpret_cast<T*>(smem_raw);
    T* lo = hi + NC * TN;
    T* rec = lo + (COMP ? NC * TN : 0);
    int* gcount = reinterpret_cast<int*>(rec + NB * RS);
    int* gstart = gcount + NG;
    int* order = gstart + NG + 1;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nactive = totals[0];
    const bool apic = s.transfer == TB_TRANSFER_APIC;
    const T dinv = T(4) / (M.h * M.h);

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
        for (int t = tid; t < NC * TN; t += NB) {
            hi[t] = T(0);
            if constexpr (COMP) lo[t] = T(0);
        }
        const int s0 = offsets[b], s1 = offsets[b + 1];
        for (int b0 = s0; b0 < s1; b0 += NB) {
            const int nbat = min(NB, s1 - b0);
            for (int g = tid; g < NG; g += NB) gcount[g] = 0;
            __syncthreads();
            // ---- 1. records + group histogram
            int grp = -1, rank = 0;
            if (tid < nbat) {
                const long long p = perm[b0 + tid] - 1;
                T x[3];
#pragma unroll
                for (int d = 0; d < D; ++d) x[d] = P.x[d][p];
                const T l = P.l ? P.l[p] : s.gimp_l;
                Basis<D, T> B;
                if (prepare_basis<D, T, GEN>(M, s.basis, x, l, B, err)) {
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
                    } else {
                        grp = gi;
                        T* r = rec + tid * RS;
                        const T Vp = P.V[p];
                        r[0] = P.m ? P.m[p] : s.mass;
#pragma unroll
                        for (int d = 0; d < D; ++d) r[1 + d] = P.v[d][p];
#pragma unroll
                        for (int k = 0; k < R::NS; ++k) r[4 + k] = (-Vp) * P.sig[k][p];
#pragma unroll
                        for (int d = 0; d < D; ++d)
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                r[R::AX + 6 * d + 2 * k] = B.ax[d].val[k];
                                r[R::AX + 6 * d + 2 * k + 1] = B.ax[d].der[k];
                            }
                        if constexpr (GEN) {
#pragma unroll
                            for (int d = 0; d < D; ++d) r[R::XP + d] = x[d];
#pragma unroll
                            for (int i = 0; i < D + 1; ++i)
#pragma unroll
                                for (int j = 0; j < D + 1; ++j)
                                    r[R::MI + i * (D + 1) + j] = B.wls ? B.Mi[i][j] : T(i == j ? 1 : 0);
                            r[R::MI + 0] = B.wls ? B.Mi[0][0] : T(-1);  // -1 marks a plain kernel
#pragma unroll
                            for (int k = 0; k < D * D; ++k) r[R::BP + k] = apic ? P.B[k][p] : T(0);
                        }
                        rank = atomicAdd(&gcount[grp], 1);
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
            if (grp >= 0) order[gstart[grp] + rank] = tid;
            __syncthreads();
            // ---- 2. one warp per group, lanes over window nodes
            const int slot = lane % NSLOT, sub = lane / NSLOT;
            const int si = slot % 3, sj = (slot / 3) % 3, sk = (D == 3) ? slot / 9 : 0;
            for (int g = warp; g < NG; g += NW) {
                const int q0 = gstart[g], q1 = gstart[g + 1];
                if (q0 == q1) continue;
                int gl[3];
                {
                    int r = g;
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        gl[d] = r % G1;
                        r /= G1;
                    }
                }
                T acc[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) acc[c] = T(0);
                T X[3] = {T(0), T(0), T(0)};
                if constexpr (GEN) {
                    X[0] = node_coord(M, 0, org[0] + gl[0] + si);
                    X[1] = node_coord(M, 1, org[1] + gl[1] + sj);
                    if constexpr (D == 3) X[2] = node_coord(M, 2, org[2] + gl[2] + sk);
                }
                if (sub < NSUB) {
                    for (int q = q0 + sub; q < q1; q += NSUB) {
                        const T* r = rec + order[q] * RS;
                        const T mp = r[0];
                        T v[3], S[6];
#pragma unroll
                        for (int d = 0; d < D; ++d) v[d] = r[1 + d];
#pragma unroll
                        for (int k = 0; k < R::NS; ++k) S[k] = r[4 + k];
                        const T wx = r[R::AX + 2 * si], dx = r[R::AX + 2 * si + 1];
                        const T wy = r[R::AX + 6 + 2 * sj], dy = r[R::AX + 6 + 2 * sj + 1];
                        T w, gw[3];
                        if constexpr (D == 3) {
                            const T wz = r[R::AX + 12 + 2 * sk], dz = r[R::AX + 12 + 2 * sk + 1];
                            w = (wx * wy) * wz;
                            gw[0] = ((dx * wy) * wz) * M.h_inv;
                            gw[1] = ((wx * dy) * wz) * M.h_inv;
                            gw[2] = ((wx * wy) * dz) * M.h_inv;
                        } else {
                            w = wx * wy;
                            gw[0] = (dx * wy) * M.h_inv;
                            gw[1] = (wx * dy) * M.h_inv;
                        }
                        if constexpr (GEN) {
                            T rel[3];
#pragma unroll
                            for (int d = 0; d < D; ++d) rel[d] = X[d] - r[R::XP + d];
                            if (r[R::MI] != T(-1)) {  // WLS: wq = w Mi [1; rel]
                                constexpr int N = D + 1;
                                T Pv[N];
                                Pv[0] = T(1);
#pragma unroll
                                for (int d = 0; d < D; ++d) Pv[d + 1] = rel[d];
                                T wq[N];
#pragma unroll
                                for (int i = 0; i < N; ++i) {
                                    T a = T(0);
#pragma unroll
                                    for (int j = 0; j < N; ++j) a += r[R::MI + i * N + j] * Pv[j];
                                    wq[i] = w * a;
                                }
                                w = wq[0];
#pragma unroll
                                for (int d = 0; d < D; ++d) gw[d] = wq[d + 1];
                            }
                            if (apic) {
#pragma unroll
                                for (int i = 0; i < D; ++i) {
                                    T a = T(0);
#pragma unroll
                                    for (int j = 0; j < D; ++j) a += r[R::BP + i + j * D] * dinv * rel[j];
                                    v[i] += a;
                                }
                            }
                        }
                        const T wm = w * mp;
                        acc[0] += wm;
#pragma unroll
                        for (int d = 0; d < D; ++d) acc[1 + d] += wm * v[d];
#pragma unroll
                        for (int i = 0; i < D; ++i) {
                            T a = T(0);
#pragma unroll
                            for (int j = 0; j < D; ++j) a += S[symidx<D>(i, j)] * gw[j];
                            acc[1 + D + i] += a;
                        }
                    }
                }
                if constexpr (NSUB > 1) {
#pragma unroll
                    for (int u = 1; u < NSUB; ++u)
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            const T o = __shfl_sync(0xffffffffu, acc[c], min(lane + u * NSLOT, 31));
                            if (sub == 0) acc[c] += o;
                        }
                }
                if (sub == 0) {
                    const int ti = gl[0] + si, tj = gl[1] + sj, tk = (D == 3) ? gl[D - 1] + sk : 0;
                    const int t = (D == 3) ? ti + TS * (tj + TS * tk) : ti + TS * tj;
#pragma unroll
                    for (int c = 0; c < NC; ++c) tile_add(hi, lo, c * TN + t, acc[c]);
                }
            }
            __syncthreads();
        }
        // ---- 3. flush the tile
        for (int t = tid; t < TN; t += NB) {
            int node[3], rem = t;
            bool inside = true;
            long long lin = 0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                node[d] = org[d] + rem % TS;
                rem /= TS;
                inside = inside && node[d] >= 0 && node[d] < M.n[d];
            }
            if (!inside) continue;
#pragma unroll
            for (int d = D - 1; d >= 0; --d) lin = lin * M.n[d] + node[d];
            T val[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                val[c] = hi[c * TN + t];
                if constexpr (COMP) val[c] += lo[c * TN + t];
            }
#pragma unroll
            for (int d = 0; d < D; ++d) val[1 + D + d] += s.g[d] * val[0];
            if (val[0] != T(0)) atomicAdd(G.m + lin, val[0]);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                if (val[1 + d] != T(0)) atomicAdd(G.mv[d] + lin, val[1 + d]);
                if (val[1 + D + d] != T(0)) atomicAdd(G.f[d] + lin, val[1 + D + d]);
            }
        }
        __syncthreads();
    }
}

template <int D, class T, int BW, bool GEN, int NB>
size_t p2g_smem_bytes() {
    constexpr int TS = BW + 3;
    constexpr int TN = (D == 3) ? TS * TS * TS : TS * TS;
    constexpr int NC = 1 + 2 * D;
    constexpr int NG = (D == 3) ? (BW + 1) * (BW + 1) * (BW + 1) : (BW + 1) * (BW + 1);
    const size_t tiles = sizeof(T) * size_t(NC * TN) * (sizeof(T) == 4 ? 2 : 1);
    const size_t recs = sizeof(T) * size_t(NB) * Rec<D, GEN>::SIZE;
    const size_t ints = sizeof(int) * size_t(NG + NG + 1 + NB);
    return tiles + recs + ints;
}

template <int D, class T, int BW, bool GEN>
cudaError_t launch_group(const DMesh<D, T>& M, const PView<T>& P, const GView<T>& G, const Scalars<T>& s,
                         const BinBuffers& b, const LaunchCfg& cfg) {
    constexpr int NB = 256;
    auto kern = p2g_group_kernel<D, T, BW, GEN, NB>;
    const size_t smem = p2g_smem_bytes<D, T, BW, GEN, NB>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NB, smem);
    const int grid = std::min(cfg.num_sms * std::max(per_sm, 1), M.nblocks);
    kern<<<grid, NB, smem, cfg.stream>>>(M, P, G, s, b.totals, b.blocklist, b.offsets, b.perm, cfg.err);
    ++*cfg.launches;
    return cudaGetLastError();
}

}  // namespace

template <int D, class T, int BW>
cudaError_t launch_p2g(const DMesh<D, T>& M, const PView<T>& P, const GView<T>& G, const Scalars<T>& s,
                       const BinBuffers& b, const LaunchCfg& cfg) {
    cudaError_t e = launch_grid_zero<D, T>(M, G, cfg);
    if (e != cudaSuccess) return e;
    if (P.n == 0) return cudaSuccess;
    const bool gen = s.transfer == TB_TRANSFER_APIC || s.basis == TB_WLS_BSPLINE_QUADRATIC || s.basis == TB_WLS_UGIMP;
    return gen ? launch_group<D, T, BW, true>(M, P, G, s, b, cfg) : launch_group<D, T, BW, false>(M, P, G, s, b, cfg);
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
