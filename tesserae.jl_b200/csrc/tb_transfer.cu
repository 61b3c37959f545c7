// tb_transfer.cu -- grid update and G2P kernels of the explicit MPM step.
//
// (P2G is in tb_p2g.cu.)
// grid (src/Transfer/foreach.jl:276-339, docs/src/gpu.md:309-316): vn = mv/m,
//      v = vn + dt f / m guarded by m != 0, then the slip-wall slices.
// G2P  (src/Transfer/gpu.jl:226-232, README.md:79-86): one CTA per non-empty
//      block stages the block's (v, v - vn) tile in shared memory and gathers
//      for each particle of the block (3D FP32: packed FP32x2 FMAs over the
//      component pairs of a node-major tile); particles outside the mesh (empty
//      window) are updated by a particle-parallel pass.
#include "tb_launch.cuh"

namespace tb {

namespace {

template <int D, int BW>
struct Tile {
    static constexpr int TS = BW + 3;
    static constexpr int TN = (D == 3) ? TS * TS * TS : TS * TS;
};

template <int D, class T>
__device__ __forceinline__ void load_x(const PView<T>& P, long long p, T* x) {
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] = P.x[d][p];
}

// Stored nodes of a grid: every node of a dense grid; the active blocks' nodes
// (up to the fields' capacity) of a sparse one.
template <int D, class T>
__device__ __forceinline__ long long stored_nodes(const GView<T>& G, long long nnodes) {
    if (!G.bnum) return nnodes;
    const long long n = (long long)G.nact[0] << (G.L * D);
    return n < G.cap ? n : G.cap;
}

template <int D, class T>
__global__ void __launch_bounds__(256) grid_zero_kernel(GView<T> G, long long nnodes) {
    const long long nn = stored_nodes<D>(G, nnodes);
    for (long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x; I < nn; I += (long long)gridDim.x * blockDim.x) {
        G.m[I] = T(0);
#pragma unroll
        for (int d = 0; d < D; ++d) {
            G.mv[d][I] = T(0);
            G.f[d][I] = T(0);
        }
    }
}

template <int D, class T>
__global__ void __launch_bounds__(256) grid_update_kernel(DMesh<D, T> M, GView<T> G, Scalars<T> s) {
    const long long nn = stored_nodes<D>(G, M.nnodes);
    for (long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x; I < nn;
         I += (long long)gridDim.x * blockDim.x) {
        int idx[3] = {0, 0, 0};
        if (G.bnum) {
            // slot I of storage block k: node (B's origin) + (column-major local index)
            const int W = 1 << G.L, k = int(I >> (G.L * D)), q = int(I & ((1ll << (G.L * D)) - 1));
            const int B = G.blist[k] - 1;
            const int bidx[3] = {B % M.nb[0], (B / M.nb[0]) % M.nb[1], D == 3 ? B / (M.nb[0] * M.nb[1]) : 0};
            const int qidx[3] = {q % W, (q / W) % W, q / (W * W)};
            bool inside = true;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                idx[d] = bidx[d] * W + qidx[d];
                inside = inside && idx[d] < M.n[d];
            }
            if (!inside) {  // a block's nodes past the mesh edge
#pragma unroll
                for (int d = 0; d < D; ++d) G.vn[d][I] = G.v[d][I] = T(0);
                continue;
            }
        } else {
            long long r = I;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                idx[d] = int(r % M.n[d]);
                r /= M.n[d];
            }
        }
        const T m = G.m[I];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            T vn = T(0), v = T(0);
            if (m != T(0)) {
                vn = G.mv[d][I] / m;
                v = vn + (s.dt * G.f[d][I]) / m;
            }
            if (s.wall_mask) {
                const bool lo = (s.wall_mask >> (2 * d)) & 1, hi = (s.wall_mask >> (2 * d + 1)) & 1;
                if ((lo && idx[d] < s.wall_layers) || (hi && idx[d] >= M.n[d] - s.wall_layers)) {
                    vn = T(0);
                    v = T(0);
                }
            }
            G.vn[d][I] = vn;
            G.v[d][I] = v;
        }
    }
}

// ---- sparse grid maintenance -------------------------------------------
// Node block B owns nodes [BW B, BW B + BW - 1] per axis. A particle block b
// reaches nodes [BW b - 1, BW b + BW + 1], i.e. node blocks b-1 .. b+1 per axis.
template <int D>
__global__ void __launch_bounds__(128) mark_touched_kernel(const int* __restrict__ totals,
                                                           const int* __restrict__ blocklist, int3 nb,
                                                           unsigned char* __restrict__ cur) {
    const int nactive = totals[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nactive; i += gridDim.x * blockDim.x) {
        const int b = blocklist[i] - 1;
        const int bx = b % nb.x, by = (b / nb.x) % nb.y, bz = (D == 3) ? b / (nb.x * nb.y) : 0;
        for (int dz = (D == 3 ? -1 : 0); dz <= (D == 3 ? 1 : 0); ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = bx + dx, y = by + dy, z = bz + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= nb.x || y >= nb.y || (D == 3 && z >= nb.z)) continue;
                    cur[x + nb.x * (y + nb.y * z)] = 1;
                }
    }
}

// The node blocks marked in cur or prev, compacted into a list (one atomic per
// warp; the order of the list does not matter, every block is processed on its
// own), so the zero and update passes visit the touched blocks only instead of
// testing every block's flags.
__global__ void __launch_bounds__(256) touched_list_kernel(const unsigned char* __restrict__ cur,
                                                           const unsigned char* __restrict__ prev, int nblocks,
                                                           int* __restrict__ list, int* __restrict__ count) {
    const int lane = threadIdx.x & 31;
    for (int B0 = blockIdx.x * blockDim.x; B0 < nblocks; B0 += gridDim.x * blockDim.x) {
        const int B = B0 + threadIdx.x;
        const bool t = B < nblocks && (cur[B] | prev[B]);
        const unsigned m = __ballot_sync(0xffffffffu, t);
        int base = 0;
        if (lane == 0 && m) base = atomicAdd(count, __popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (t) list[base + __popc(m & ((1u << lane) - 1u))] = B;
    }
}

// One warp per listed node block. mode 0: zero m, mv, f; mode 1: grid update
// where cur, zero v, vn where the block was touched by the previous transfer only;
// with zero_after, m, mv and f of the cur blocks are zeroed once read (the next
// P2G of the same call then needs no zero pass).
template <int D, class T, int BW, int MODE>
__global__ void __launch_bounds__(256) node_list_kernel(DMesh<D, T> M, GView<T> G, Scalars<T> s,
                                                        const unsigned char* __restrict__ cur,
                                                        const int* __restrict__ list, const int* __restrict__ count,
                                                        int zero_after) {
    constexpr int NPB = (D == 3) ? BW * BW * BW : BW * BW;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int nlist = *count;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nlist; w += warps) {
        const int B = list[w];
        const bool c = MODE == 1 ? cur[B] != 0 : true;
        const int bx = B % M.nb[0], by = (B / M.nb[0]) % M.nb[1], bz = (D == 3) ? B / (M.nb[0] * M.nb[1]) : 0;
        for (int q = lane; q < NPB; q += 32) {
            int idx[3];
            idx[0] = bx * BW + q % BW;
            idx[1] = by * BW + (q / BW) % BW;
            idx[2] = (D == 3) ? bz * BW + q / (BW * BW) : 0;
            bool inside = true;
#pragma unroll
            for (int d = 0; d < D; ++d) inside = inside && idx[d] < M.n[d];
            if (!inside) continue;
            long long I = 0;
#pragma unroll
            for (int d = D - 1; d >= 0; --d) I = I * M.n[d] + idx[d];
            if constexpr (MODE == 0) {
                G.m[I] = T(0);
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    G.mv[d][I] = T(0);
                    G.f[d][I] = T(0);
                }
            } else {
                const T m = c ? G.m[I] : T(0);
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    T vn = T(0), v = T(0);
                    if (m != T(0)) {
                        vn = G.mv[d][I] / m;
                        v = vn + (s.dt * G.f[d][I]) / m;
                    }
                    if (s.wall_mask) {
                        const bool lo = (s.wall_mask >> (2 * d)) & 1, hi = (s.wall_mask >> (2 * d + 1)) & 1;
                        if ((lo && idx[d] < s.wall_layers) || (hi && idx[d] >= M.n[d] - s.wall_layers)) {
                            vn = T(0);
                            v = T(0);
                        }
                    }
                    G.vn[d][I] = vn;
                    G.v[d][I] = v;
                }
                if (zero_after && c) {
                    G.m[I] = T(0);
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        G.mv[d][I] = T(0);
                        G.f[d][I] = T(0);
                    }
                }
            }
        }
    }
}

// Final per-particle writes of @G2P and the FP64 constitutive update.
template <int D, class T, bool VM = false>
__device__ __forceinline__ void g2p_finish(const PView<T>& P, const Scalars<T>& s, long long p, const T* x,
                                           const T* vp, const T* vpic, const T* dvf, const T (&gv)[3][3],
                                           const T* dxs, const T (&Bn)[3][3], const double (&F)[3][3]) {
    if (s.transfer == TB_TRANSFER_APIC) {
#pragma unroll
        for (int d = 0; d < D; ++d) P.v[d][p] = vpic[d];
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) P.B[r + c * D][p] = Bn[r][c];
    } else {
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const T vflip = vp[d] + dvf[d];
            P.v[d][p] = (s.alpha == T(1)) ? vflip : (T(1) - s.alpha) * vpic[d] + s.alpha * vflip;
        }
    }
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
        for (int c = 0; c < D; ++c) P.gv[r + c * D][p] = gv[r][c];
    if (P.x[0]) {  // the FP64-position form writes x itself
#pragma unroll
        for (int d = 0; d < D; ++d) (P.x_out[0] ? P.x_out[d] : P.x[d])[p] = x[d] + dxs[d];
    }
    particle_update<D, T, VM>(P, s, p, gv, F);
}

template <int D, class T, int BW, bool GEN, bool X64, bool VM = false>
__global__ void __launch_bounds__(128, (GEN || VM) ? (sizeof(T) == 4 ? 4 : 2) : (sizeof(T) == 4 ? 8 : 4)) g2p_tile_kernel(DMesh<D, T> M, GView<T> G, PView<T> P, Scalars<T> s,
                                                       const int* __restrict__ totals,
                                                       const int* __restrict__ blocklist,
                                                       const int* __restrict__ offsets,
                                                       const int* __restrict__ perm, int* err,
                                                       int* __restrict__ next_bid, int* __restrict__ next_count) {
    constexpr int TS = Tile<D, BW>::TS, TN = Tile<D, BW>::TN;
    // 3D FP32: node-major, (v_x, v_y, v_z, dv_x) as a float4 at [t] and (dv_y, dv_z)
    // as a float2 after the TN float4s, dv = v - vn: two vector loads per node,
    // whose halves feed packed FP32x2 FMAs. Otherwise component-major: v_r at
    // [r TN + t], dv_r at [(D + r) TN + t]; lanes reading different nodes hit
    // different banks.
    constexpr bool VEC = (D == 3 && sizeof(T) == 4);
    __shared__ __align__(16) T tile[2 * D * TN];
    auto node_vals = [&](int t, T (&vi)[3], T (&dvi)[3]) {
        if constexpr (VEC) {
            const float4 a = reinterpret_cast<const float4*>(tile)[t];
            const float2 c = reinterpret_cast<const float2*>(tile + 4 * TN)[t];
            vi[0] = a.x; vi[1] = a.y; vi[2] = a.z;
            dvi[0] = a.w; dvi[1] = c.x; dvi[2] = c.y;
        } else {
#pragma unroll
            for (int d = 0; d < D; ++d) {
                vi[d] = tile[d * TN + t];
                dvi[d] = tile[(D + d) * TN + t];
            }
        }
    };
    const int nactive = totals[0];
    const int tid = threadIdx.x, nth = blockDim.x;
    const bool apic = s.transfer == TB_TRANSFER_APIC;
    // CTA `piece` of `split` sharing a block takes its particles piece nth + tid,
    // (piece + split) nth + tid, ... (block_split: 4 particles per thread)
    const int split = block_split(totals, 4 * nth);
    const int stride = split * nth;
    for (int vi = blockIdx.x; vi < nactive * split; vi += gridDim.x) {
        const int bi = split == 1 ? vi : vi / split, piece = vi - bi * split;
        int b = blocklist[bi] - 1;
        int org[3] = {0, 0, 0};
#pragma unroll
        for (int d = 0; d < D; ++d) {
            org[d] = (b % M.nb[d]) * BW - 1;
            b /= M.nb[d];
        }
        b = blocklist[bi] - 1;
        // the block's particle range and this thread's first particle id are
        // loaded before the tile, so their round trips overlap the tile's
        const int s0 = offsets[b] + piece * nth, s1 = offsets[b + 1];
        int pnext = (s0 + tid < s1) ? perm[s0 + tid] : 1;
        for (int t = tid; t < TN; t += nth) {
            int node[3] = {0, 0, 0}, rem = t;
            bool inside = true;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                node[d] = org[d] + rem % TS;
                rem /= TS;
                inside = inside && node[d] >= 0 && node[d] < M.n[d];
            }
            // nodes outside the mesh, and nodes a sparse grid does not store, read as zero
            const long long sl = inside ? grid_slot<D>(G, M, node[0], node[1], node[2]) : -1;
            T vi[3] = {T(0), T(0), T(0)}, dvi[3] = {T(0), T(0), T(0)};
#pragma unroll
            for (int d = 0; d < D; ++d) {
                vi[d] = sl >= 0 ? G.v[d][sl] : T(0);
                const T vni = sl >= 0 ? G.vn[d][sl] : T(0);
                dvi[d] = vi[d] - vni;
            }
            if constexpr (VEC) {
                reinterpret_cast<float4*>(tile)[t] = make_float4(vi[0], vi[1], vi[2], dvi[0]);
                reinterpret_cast<float2*>(tile + 4 * TN)[t] = make_float2(dvi[1], dvi[2]);
            } else {
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    tile[d * TN + t] = vi[d];
                    tile[(D + d) * TN + t] = dvi[d];
                }
            }
        }
        __syncthreads();
        for (int j = s0 + tid; j < s1; j += stride) {
            const long long p = pnext - 1;
            pnext = (j + stride < s1) ? perm[j + stride] : 1;  // next id in flight during this particle
            T x[3] = {T(0), T(0), T(0)}, vp[3];
            double xd[3] = {0.0, 0.0, 0.0};
            if constexpr (X64) {
#pragma unroll
                for (int d = 0; d < D; ++d) xd[d] = P.x64[d][p];
            } else {
                load_x<D, T>(P, p, x);
            }
#pragma unroll
            for (int d = 0; d < D; ++d) vp[d] = P.v[d][p];
            // F (72 bytes in FP64): the FP32 B-spline/uGIMP kernel (64 registers)
            // loads it after the gather, where holding it across the gather cost
            // spills (G2P 1.032 -> 1.019 ms on cube3d); the FP64 and WLS/APIC
            // kernels load it here so that the load overlaps the gather (loading
            // it late measured 7% and 1% slower there).
            constexpr bool LATE_F = !GEN && sizeof(T) == 4;
            double F[3][3];
            if constexpr (!LATE_F) load_F<D, T>(P, p, F);
            const T l = P.l ? P.l[p] : s.gimp_l;
            T vpic[3] = {T(0), T(0), T(0)}, dvf[3] = {T(0), T(0), T(0)}, dxs[3] = {T(0), T(0), T(0)};
            T gv[3][3] = {}, Bn[3][3] = {};
            Basis<D, T> B;
            bool in;
            if constexpr (X64) in = prepare_basis_x64<D, T, GEN>(M, s.basis, xd, l, B, err);
            else in = prepare_basis<D, T, GEN>(M, s.basis, x, l, B, err);
            if (in) {
                int q0[3] = {0, 0, 0};
                bool ok = true;
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    q0[d] = B.ax[d].lo - org[d];
                    ok = ok && q0[d] >= 0 && q0[d] + 2 < TS;
                }
                if (!ok) {
                    atomicOr(err, ERR_TILE_RANGE);
                } else if constexpr (!GEN && VEC) {
                    // The separable contraction below with the component pairs of the
                    // node-major tile in packed FP32x2 FMAs; every lane of a pair is
                    // the scalar form's FMA with the same operands in the same order.
                    float gx[3];
#pragma unroll
                    for (int i = 0; i < 3; ++i) gx[i] = B.ax[0].der[i] * M.h_inv;
                    const float4* tA = reinterpret_cast<const float4*>(tile);
                    const float2* tB = reinterpret_cast<const float2*>(tile + 4 * TN);
                    const float2 z2 = make_float2(0.f, 0.f);
                    // (vpic_x, vpic_y), (vpic_z, dvf_x), (dvf_y, dvf_z), (gv_xc, gv_yc) per column c, gv_zc
                    float2 p01 = z2, p2d0 = z2, d12 = z2, g0 = z2, g1 = z2, g2 = z2;
                    float g0z = 0.f, g1z = 0.f, g2z = 0.f;
#pragma unroll
                    for (int k = 0; k < 3; ++k)
#pragma unroll
                        for (int jj = 0; jj < 3; ++jj) {
                            float2 Av01 = z2, Av2d0 = z2, Ad12 = z2, Ag01 = z2;
                            float Ag2 = 0.f;
                            const int t0 = q0[0] + TS * ((q0[1] + jj) + TS * (q0[2] + k));
#pragma unroll
                            for (int i = 0; i < 3; ++i) {
                                const float4 a = tA[t0 + i];
                                const float2 c = tB[t0 + i];
                                const float2 v01 = make_float2(a.x, a.y);
                                const float2 wxx = make_float2(B.ax[0].val[i], B.ax[0].val[i]);
                                const float2 gxx = make_float2(gx[i], gx[i]);
                                Av01 = __ffma2_rn(wxx, v01, Av01);
                                Av2d0 = __ffma2_rn(wxx, make_float2(a.z, a.w), Av2d0);
                                Ad12 = __ffma2_rn(wxx, c, Ad12);
                                Ag01 = __ffma2_rn(gxx, v01, Ag01);
                                Ag2 = __fmaf_rn(gx[i], a.z, Ag2);
                            }
                            const float wyz = B.ax[1].val[jj] * B.ax[2].val[k];
                            const float dyz = (B.ax[1].der[jj] * M.h_inv) * B.ax[2].val[k];
                            const float wdz = B.ax[1].val[jj] * (B.ax[2].der[k] * M.h_inv);
                            const float2 W = make_float2(wyz, wyz), DY = make_float2(dyz, dyz),
                                         DZ = make_float2(wdz, wdz);
                            p01 = __ffma2_rn(W, Av01, p01);
                            p2d0 = __ffma2_rn(W, Av2d0, p2d0);
                            d12 = __ffma2_rn(W, Ad12, d12);
                            g0 = __ffma2_rn(W, Ag01, g0);
                            g0z = __fmaf_rn(wyz, Ag2, g0z);
                            g1 = __ffma2_rn(DY, Av01, g1);
                            g1z = __fmaf_rn(dyz, Av2d0.x, g1z);
                            g2 = __ffma2_rn(DZ, Av01, g2);
                            g2z = __fmaf_rn(wdz, Av2d0.x, g2z);
                        }
                    vpic[0] = p01.x; vpic[1] = p01.y; vpic[2] = p2d0.x;
                    dvf[0] = p2d0.y; dvf[1] = d12.x; dvf[2] = d12.y;
                    gv[0][0] = g0.x; gv[1][0] = g0.y; gv[2][0] = g0z;
                    gv[0][1] = g1.x; gv[1][1] = g1.y; gv[2][1] = g1z;
                    gv[0][2] = g2.x; gv[1][2] = g2.y; gv[2][2] = g2z;
#pragma unroll
                    for (int d = 0; d < D; ++d) dxs[d] = vpic[d] * s.dt;
                } else if constexpr (!GEN) {
                    // Separable contraction: sum over the x-slot first, then weight
                    // the partial sums with the y (and z) factors.
                    T dxh[3];
#pragma unroll
                    for (int i = 0; i < 3; ++i) dxh[i] = B.ax[0].der[i] * M.h_inv;
#pragma unroll
                    for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
#pragma unroll
                        for (int jj = 0; jj < 3; ++jj) {
                            T Av[3] = {T(0), T(0), T(0)}, Adv[3] = {T(0), T(0), T(0)}, Ag[3] = {T(0), T(0), T(0)};
                            const int t0 = (D == 3) ? q0[0] + TS * ((q0[1] + jj) + TS * (q0[D - 1] + k))
                                                    : q0[0] + TS * (q0[1] + jj);
#pragma unroll
                            for (int i = 0; i < 3; ++i) {
                                const T* nd = tile + (t0 + i);
                                const T wx = B.ax[0].val[i], gx = dxh[i];
#pragma unroll
                                for (int r = 0; r < D; ++r) {
                                    const T vi = nd[r * TN], dvi = nd[(D + r) * TN];
                                    Av[r] += wx * vi;
                                    Adv[r] += wx * dvi;
                                    Ag[r] += gx * vi;
                                }
                            }
                            T wyz, dyz, wdz;
                            if constexpr (D == 3) {
                                wyz = B.ax[1].val[jj] * B.ax[D - 1].val[k];
                                dyz = (B.ax[1].der[jj] * M.h_inv) * B.ax[D - 1].val[k];
                                wdz = B.ax[1].val[jj] * (B.ax[D - 1].der[k] * M.h_inv);
                            } else {
                                wyz = B.ax[1].val[jj];
                                dyz = B.ax[1].der[jj] * M.h_inv;
                                wdz = T(0);
                            }
#pragma unroll
                            for (int r = 0; r < D; ++r) {
                                vpic[r] += wyz * Av[r];
                                dvf[r] += wyz * Adv[r];
                                gv[r][0] += wyz * Ag[r];
                                gv[r][1] += dyz * Av[r];
                                if constexpr (D == 3) gv[r][2] += wdz * Av[r];
                            }
                        }
#pragma unroll
                    for (int d = 0; d < D; ++d) dxs[d] = vpic[d] * s.dt;
                } else {
                    // WLS / APIC: node weights are not separable; per-node loop.
#pragma unroll
                    for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
#pragma unroll
                        for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                            for (int i = 0; i < 3; ++i) {
                                const int idx[3] = {i, jj, k};
                                const int t = (D == 3) ? (q0[0] + i) + TS * ((q0[1] + jj) + TS * (q0[D - 1] + k))
                                                       : (q0[0] + i) + TS * (q0[1] + jj);
                                T rel[3] = {T(0), T(0), T(0)};
#pragma unroll
                                for (int d = 0; d < D; ++d) {
                                    if constexpr (X64)  // X_i - x_p in FP64, rounded once
                                        rel[d] = T(__dadd_rn(M.xmin64[d], __dmul_rn(double(B.ax[d].lo + idx[d]), M.h64)) -
                                                   xd[d]);
                                    else
                                        rel[d] = node_coord(M, d, B.ax[d].lo + idx[d]) - x[d];
                                }
                                T w, dw[3];
                                eval_node<D, T>(M, B, i, jj, k, rel, w, dw);
                                T vi[3], dvi[3];
                                node_vals(t, vi, dvi);
#pragma unroll
                                for (int d = 0; d < D; ++d) {
                                    vpic[d] += w * vi[d];
                                    dvf[d] += w * dvi[d];
                                    dxs[d] += (w * vi[d]) * s.dt;
                                }
#pragma unroll
                                for (int r = 0; r < D; ++r)
#pragma unroll
                                    for (int c = 0; c < D; ++c) gv[r][c] += vi[r] * dw[c];
                                if (apic) {
#pragma unroll
                                    for (int r = 0; r < D; ++r)
#pragma unroll
                                        for (int c = 0; c < D; ++c) Bn[r][c] += (w * vi[r]) * rel[c];
                                }
                            }
                }
            }
            if constexpr (LATE_F) load_F<D, T>(P, p, F);
            g2p_finish<D, T, VM>(P, s, p, x, vp, vpic, dvf, gv, dxs, Bn, F);
            int nb = 0;
            if constexpr (X64) {
                double xn[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    xn[d] = xd[d] + double(dxs[d]);
                    (P.x64_out[0] ? P.x64_out[d] : P.x64[d])[p] = xn[d];
                }
                if (next_bid) nb = findblock_x64<D, T>(M, xn);
            } else {
                if (next_bid) {
                    T xn[3] = {T(0), T(0), T(0)};
#pragma unroll
                    for (int d = 0; d < D; ++d) xn[d] = x[d] + dxs[d];  // the value g2p_finish stored
                    nb = findblock<D, T>(M, xn);
                }
            }
            if (next_bid) {
                // the next step's count pass: warp-aggregated, as bin_count_kernel
                next_bid[p] = nb;
                const unsigned act = __activemask();
                const unsigned peers = __match_any_sync(act, nb);
                if (nb > 0 && int(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&next_count[nb - 1], __popc(peers));
            }
        }
        __syncthreads();
    }
}

// Particle-parallel G2P reading the grid from global memory: the reference's own
// G2P schedule (one thread per particle, gpu.jl:226-232); needs no partition.
template <int D, class T, bool VM = false>
__global__ void __launch_bounds__(128) g2p_direct_kernel(DMesh<D, T> M, GView<T> G, PView<T> P, Scalars<T> s,
                                                         int* err) {
    const bool apic = s.transfer == TB_TRANSFER_APIC;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P.n; p += (long long)gridDim.x * blockDim.x) {
        T x[3], vp[3];
        load_x<D, T>(P, p, x);
#pragma unroll
        for (int d = 0; d < D; ++d) vp[d] = P.v[d][p];
        double F[3][3];
        load_F<D, T>(P, p, F);
        const T l = P.l ? P.l[p] : s.gimp_l;
        T vpic[3] = {T(0), T(0), T(0)}, dvf[3] = {T(0), T(0), T(0)}, dxs[3] = {T(0), T(0), T(0)};
        T gv[3][3] = {}, Bn[3][3] = {};
        Basis<D, T> B;
        if (prepare_basis<D, T>(M, s.basis, x, l, B, err)) {
            const bool need_rel = B.wls || apic;
#pragma unroll
            for (int k = 0; k < (D == 3 ? 3 : 1); ++k)
#pragma unroll
                for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const int idx[3] = {i, jj, k};
                        long long lin = 0;
                        bool valid = true;
#pragma unroll
                        for (int d = D - 1; d >= 0; --d) valid = valid && idx[d] < B.ax[d].cnt;
                        if (valid) {
                            lin = grid_slot<D>(G, M, B.ax[0].lo + idx[0], B.ax[1].lo + idx[1],
                                               D == 3 ? B.ax[D - 1].lo + idx[D - 1] : 0);
                            valid = lin >= 0;
                        }
                        T rel[3] = {T(0), T(0), T(0)};
                        if (need_rel) {
#pragma unroll
                            for (int d = 0; d < D; ++d) rel[d] = node_coord(M, d, B.ax[d].lo + idx[d]) - x[d];
                        }
                        T w, dw[3];
                        eval_node<D, T>(M, B, i, jj, k, rel, w, dw);
                        T vi[3];
#pragma unroll
                        for (int d = 0; d < D; ++d) {
                            vi[d] = valid ? __ldg(G.v[d] + lin) : T(0);
                            const T dv = valid ? vi[d] - __ldg(G.vn[d] + lin) : T(0);
                            vpic[d] += w * vi[d];
                            dvf[d] += w * dv;
                            dxs[d] += (w * vi[d]) * s.dt;
                        }
#pragma unroll
                        for (int r = 0; r < D; ++r)
#pragma unroll
                            for (int c = 0; c < D; ++c) gv[r][c] += vi[r] * dw[c];
                        if (apic) {
#pragma unroll
                            for (int r = 0; r < D; ++r)
#pragma unroll
                                for (int c = 0; c < D; ++c) Bn[r][c] += (w * vi[r]) * rel[c];
                        }
                    }
        }
        g2p_finish<D, T, VM>(P, s, p, x, vp, vpic, dvf, gv, dxs, Bn, F);
    }
}

// Particles outside the mesh (block id 0): empty window, so only the particle
// equations run (v and x keep their values under FLIP).
template <int D, class T, bool VM = false>
__global__ void __launch_bounds__(256) g2p_outside_kernel(PView<T> P, Scalars<T> s, const int* __restrict__ blockids,
                                                          const int* __restrict__ totals) {
    if ((long long)totals[1] >= P.n) return;  // every particle is inside a block
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P.n; p += (long long)gridDim.x * blockDim.x) {
        if (blockids[p] != 0) continue;
        T x[3], vp[3], z[3] = {T(0), T(0), T(0)};
        T gv[3][3] = {}, Bn[3][3] = {};
#pragma unroll
        for (int d = 0; d < D; ++d) {
            x[d] = P.x[0] ? P.x[d][p] : T(0);  // FP64 positions stay as they are
            vp[d] = P.v[d][p];
        }
        double F[3][3];
        load_F<D, T>(P, p, F);
        g2p_finish<D, T, VM>(P, s, p, x, vp, z, z, gv, z, Bn, F);
    }
}

// c = sqrt((lambda + 2 mu) / (m / V)) + |v| per particle, the Taylor impact's
// speed for its time step (docs/src/gpu.md:283-284); the maximum goes to *out
// as the bits of a non-negative double, which order as unsigned integers.
template <int D, class T>
__global__ void __launch_bounds__(256) wave_speed_kernel(PView<T> P, Scalars<T> s, unsigned long long* out) {
    double cmax = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P.n; p += (long long)gridDim.x * blockDim.x) {
        const double mu = P.mu ? double(P.mu[p]) : s.mu;
        const double lam = P.lam ? double(P.lam[p]) : s.lam;
        const double m = P.m ? double(P.m[p]) : double(s.mass);
        double vv = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) vv += double(P.v[d][p]) * double(P.v[d][p]);
        const double c = sqrt((lam + 2.0 * mu) / (m / double(P.V[p]))) + sqrt(vv);
        cmax = fmax(cmax, c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cmax = fmax(cmax, __shfl_down_sync(0xffffffffu, cmax, o));
    if ((threadIdx.x & 31) == 0 && cmax > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(cmax));
}

// update!(weights, particles, mesh) with stored values (basis_weight.jl:714-752):
// w in (3,3,3,n) column-major, grad_w as Vec{D} per slot, window as 1-based
// (start, stop) Int64 pairs; slots outside a truncated window are zeroed.
template <int D, class T>
__global__ void __launch_bounds__(128) update_weights_kernel(DMesh<D, T> M, PView<T> P, Scalars<T> s, T* w_out,
                                                             T* gw_out, long long* win_out, int* err) {
    constexpr int NW = (D == 3) ? 27 : 9;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P.n; p += (long long)gridDim.x * blockDim.x) {
        T x[3];
        load_x<D, T>(P, p, x);
        const T l = P.l ? P.l[p] : s.gimp_l;
        Basis<D, T> B;
        const bool ok = prepare_basis<D, T>(M, s.basis, x, l, B, err);
        for (int slot = 0; slot < NW; ++slot) {
            const int i = slot % 3, jj = (slot / 3) % 3, k = slot / 9;
            T w = T(0), dw[3] = {T(0), T(0), T(0)};
            if (ok && i < B.ax[0].cnt && jj < B.ax[1].cnt && (D == 2 || k < B.ax[D - 1].cnt)) {
                const int idx[3] = {i, jj, k};
                T rel[3] = {T(0), T(0), T(0)};
                if (B.wls) {
#pragma unroll
                    for (int d = 0; d < D; ++d) rel[d] = node_coord(M, d, B.ax[d].lo + idx[d]) - x[d];
                }
                eval_node<D, T>(M, B, i, jj, k, rel, w, dw);
            }
            w_out[p * NW + slot] = w;
#pragma unroll
            for (int d = 0; d < D; ++d) gw_out[(p * NW + slot) * D + d] = dw[d];
        }
#pragma unroll
        for (int d = 0; d < D; ++d) {
            win_out[p * 2 * D + 2 * d] = ok ? B.ax[d].lo + 1 : 1;
            win_out[p * 2 * D + 2 * d + 1] = ok ? B.ax[d].lo + B.ax[d].cnt : 0;
        }
    }
}

template <class K>
int occupancy_grid(K kernel, int threads, int num_sms) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
    return num_sms * (per_sm > 0 ? per_sm : 1);
}

}  // namespace

template <int D, class T>
cudaError_t launch_grid_zero(const DMesh<D, T>& M, const GView<T>& G, const LaunchCfg& cfg) {
    const long long nn = G.bnum ? G.cap : M.nnodes;  // a sparse grid's count is on the device
    const int grid = int(std::min<long long>((nn + 255) / 256, (long long)cfg.num_sms * 16));
    KernelScope ks(cfg, "grid_zero");
    grid_zero_kernel<D, T><<<grid, 256, 0, cfg.stream>>>(G, nn);
    ++*cfg.launches;
    return cudaGetLastError();
}

template <int D, class T>
cudaError_t launch_grid_update(const DMesh<D, T>& M, const GView<T>& G, const Scalars<T>& s, const LaunchCfg& cfg) {
    const long long nn = G.bnum ? G.cap : M.nnodes;  // a sparse grid's count is on the device
    const int grid = int(std::min<long long>((nn + 255) / 256, (long long)cfg.num_sms * 16));
    KernelScope ks(cfg, "grid_update");
    grid_update_kernel<D, T><<<grid, 256, 0, cfg.stream>>>(M, G, s);
    ++*cfg.launches;
    return cudaGetLastError();
}

template <int D, class T, int BW>
cudaError_t launch_g2p(const DMesh<D, T>& M, const GView<T>& G, const PView<T>& P, const Scalars<T>& s,
                       const BinBuffers& b, const LaunchCfg& cfg, bool count_next) {
    if (P.n == 0) return cudaSuccess;
    const bool gen = s.transfer == TB_TRANSFER_APIC || s.basis == TB_WLS_BSPLINE_QUADRATIC || s.basis == TB_WLS_UGIMP;
    auto kern = gen ? g2p_tile_kernel<D, T, BW, true, false> : g2p_tile_kernel<D, T, BW, false, false>;
    const bool vm = s.material == TB_MATERIAL_VONMISES;  // 3D only (checked by the caller)
    if constexpr (D == 3) {
        if (vm) kern = gen ? g2p_tile_kernel<D, T, BW, true, false, true> : g2p_tile_kernel<D, T, BW, false, false, true>;
    }
    if (P.x64[0]) {  // FP64-position form: FP32 state only (checked by the caller)
        if constexpr (sizeof(T) == 4) {
            kern = gen ? g2p_tile_kernel<D, T, BW, true, true> : g2p_tile_kernel<D, T, BW, false, true>;
            if constexpr (D == 3) {
                if (vm) kern = gen ? g2p_tile_kernel<D, T, BW, true, true, true> : g2p_tile_kernel<D, T, BW, false, true, true>;
            }
        } else {
            return cudaErrorInvalidValue;
        }
    }
    const int grid = std::min(occupancy_grid(kern, 128, cfg.num_sms), 8 * M.nblocks);  // blocks may be split
    {
        // first: it reads this step's block ids, which the tiled pass below
        // replaces with the next step's when it counts
        KernelScope ks(cfg, "g2p_outside");
        const int og = int(std::min<long long>((P.n + 255) / 256, (long long)cfg.num_sms * 8));
        if (D == 3 && s.material == TB_MATERIAL_VONMISES)
            g2p_outside_kernel<D, T, D == 3><<<og, 256, 0, cfg.stream>>>(P, s, b.blockids, b.totals);
        else
            g2p_outside_kernel<D, T><<<og, 256, 0, cfg.stream>>>(P, s, b.blockids, b.totals);
    }
    cudaError_t e = cudaSuccess;
    if (count_next) e = cudaMemsetAsync(b.counts, 0, sizeof(int) * size_t(M.nblocks), cfg.stream);
    if (e != cudaSuccess) return e;
    KernelScope ks(cfg, "g2p");
    kern<<<grid, 128, 0, cfg.stream>>>(M, G, P, s, b.totals, b.blocklist, b.offsets, b.perm, cfg.err,
                                       count_next ? b.blockids : nullptr, count_next ? b.counts : nullptr);
    *cfg.launches += 2;
    return cudaGetLastError();
}

template <int D, class T>
cudaError_t launch_g2p_direct(const DMesh<D, T>& M, const GView<T>& G, const PView<T>& P, const Scalars<T>& s,
                              const LaunchCfg& cfg) {
    if (P.n == 0) return cudaSuccess;
    const int grid = int(std::min<long long>((P.n + 127) / 128, (long long)cfg.num_sms * 32));
    KernelScope ks(cfg, "g2p_direct");
    if (D == 3 && s.material == TB_MATERIAL_VONMISES)
        g2p_direct_kernel<D, T, D == 3><<<grid, 128, 0, cfg.stream>>>(M, G, P, s, cfg.err);
    else
        g2p_direct_kernel<D, T><<<grid, 128, 0, cfg.stream>>>(M, G, P, s, cfg.err);
    ++*cfg.launches;
    return cudaGetLastError();
}

cudaError_t launch_mark_touched(int dim, const int* nbv, const BinBuffers& b, unsigned char* cur, int nblocks,
                                const LaunchCfg& cfg) {
    const int grid = std::max(1, std::min((nblocks + 127) / 128, cfg.num_sms * 8));
    const int3 nb = make_int3(nbv[0], nbv[1], nbv[2]);
    KernelScope ks(cfg, "grid_mark");
    if (dim == 3) mark_touched_kernel<3><<<grid, 128, 0, cfg.stream>>>(b.totals, b.blocklist, nb, cur);
    else mark_touched_kernel<2><<<grid, 128, 0, cfg.stream>>>(b.totals, b.blocklist, nb, cur);
    ++*cfg.launches;
    return cudaGetLastError();
}

cudaError_t launch_touched_list(const unsigned char* cur, const unsigned char* prev, int nblocks, int* list,
                                int* count, const LaunchCfg& cfg) {
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int), cfg.stream);
    if (e != cudaSuccess) return e;
    const int grid = std::max(1, std::min((nblocks + 255) / 256, cfg.num_sms * 8));
    KernelScope ks(cfg, "grid_mark");
    touched_list_kernel<<<grid, 256, 0, cfg.stream>>>(cur, prev, nblocks, list, count);
    ++*cfg.launches;
    return cudaGetLastError();
}

template <int D, class T, int BW>
cudaError_t launch_sparse_zero(const DMesh<D, T>& M, const GView<T>& G, const int* list, const int* count,
                               const LaunchCfg& cfg) {
    const int grid = int(std::max(1ll, std::min((M.nblocks * 32ll + 255) / 256, cfg.num_sms * 16ll)));
    KernelScope ks(cfg, "grid_zero");
    node_list_kernel<D, T, BW, 0><<<grid, 256, 0, cfg.stream>>>(M, G, Scalars<T>{}, nullptr, list, count, 0);
    ++*cfg.launches;
    return cudaGetLastError();
}

template <int D, class T, int BW>
cudaError_t launch_sparse_grid_update(const DMesh<D, T>& M, const GView<T>& G, const Scalars<T>& s,
                                      const unsigned char* cur, const int* list, const int* count,
                                      const LaunchCfg& cfg, bool zero_after) {
    const int grid = int(std::max(1ll, std::min((M.nblocks * 32ll + 255) / 256, cfg.num_sms * 16ll)));
    KernelScope ks(cfg, "grid_update");
    node_list_kernel<D, T, BW, 1><<<grid, 256, 0, cfg.stream>>>(M, G, s, cur, list, count, zero_after ? 1 : 0);
    ++*cfg.launches;
    return cudaGetLastError();
}

template <int D, class T>
cudaError_t launch_wave_speed(const PView<T>& P, const Scalars<T>& s, unsigned long long* out, const LaunchCfg& cfg) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), cfg.stream);
    if (e != cudaSuccess || P.n == 0) return e;
    const int grid = int(std::max<long long>(1, std::min<long long>((P.n + 255) / 256, (long long)cfg.num_sms * 8)));
    KernelScope ks(cfg, "wave_speed");
    wave_speed_kernel<D, T><<<grid, 256, 0, cfg.stream>>>(P, s, out);
    ++*cfg.launches;
    return cudaGetLastError();
}

template <int D, class T>
cudaError_t launch_update_weights(const DMesh<D, T>& M, const PView<T>& P, const Scalars<T>& s, T* w, T* gw,
                                  long long* win, const LaunchCfg& cfg) {
    if (P.n == 0) return cudaSuccess;
    const int grid = int(std::min<long long>((P.n + 127) / 128, (long long)cfg.num_sms * 16));
    KernelScope ks(cfg, "update_weights");
    update_weights_kernel<D, T><<<grid, 128, 0, cfg.stream>>>(M, P, s, w, gw, win, cfg.err);
    ++*cfg.launches;
    return cudaGetLastError();
}

#define TB_INST_T(D, T)                                                                                      \
    template cudaError_t launch_grid_update<D, T>(const DMesh<D, T>&, const GView<T>&, const Scalars<T>&,   \
                                                  const LaunchCfg&);                                         \
    template cudaError_t launch_grid_zero<D, T>(const DMesh<D, T>&, const GView<T>&, const LaunchCfg&);     \
    template cudaError_t launch_update_weights<D, T>(const DMesh<D, T>&, const PView<T>&, const Scalars<T>&, \
                                                     T*, T*, long long*, const LaunchCfg&);                  \
    template cudaError_t launch_g2p_direct<D, T>(const DMesh<D, T>&, const GView<T>&, const PView<T>&,       \
                                                 const Scalars<T>&, const LaunchCfg&);                     \
    template cudaError_t launch_wave_speed<D, T>(const PView<T>&, const Scalars<T>&, unsigned long long*,    \
                                                 const LaunchCfg&);
#define TB_INST_TB(D, T, BW)                                                                                 \
    template cudaError_t launch_sparse_zero<D, T, BW>(const DMesh<D, T>&, const GView<T>&, const int*,         \
                                                      const int*, const LaunchCfg&);                           \
    template cudaError_t launch_sparse_grid_update<D, T, BW>(const DMesh<D, T>&, const GView<T>&,              \
                                                             const Scalars<T>&, const unsigned char*,          \
                                                             const int*, const int*, const LaunchCfg&, bool);  \
    template cudaError_t launch_g2p<D, T, BW>(const DMesh<D, T>&, const GView<T>&, const PView<T>&,         \
                                              const Scalars<T>&, const BinBuffers&, const LaunchCfg&, bool);

TB_INST_T(3, double)
TB_INST_T(3, float)
TB_INST_T(2, double)
TB_INST_T(2, float)
TB_INST_TB(3, double, 4)
TB_INST_TB(3, float, 4)
TB_INST_TB(2, double, 8)
TB_INST_TB(2, float, 8)
TB_INST_TB(2, double, 4)
TB_INST_TB(2, float, 4)

}  // namespace tb
